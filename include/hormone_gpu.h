/*
 * hormone_gpu.h -- C ABI of the B200 implementation of HORMONE's explicit
 * MHD step.
 *
 * The reference has no plugin or FFI layer: its step loop
 * (src/main/hormone.f90:124-179) calls four argument-less subroutines that
 * read and write module globals.  Each entry point below replaces one of
 * them; a Fortran ISO_C_BINDING shim keeps the subroutine names and passes
 * the module arrays.  All functions return 0 on success or a negative
 * HMN_E* code, and never abort the host process.
 *
 * Layout: host arrays are Fortran order (i fastest) and may carry
 * ``ghost`` layers on every side (2 for HORMONE's module arrays
 * u(is-2:ie+2,js-2:je+2,ks-2:ke+2,1:ufnmax), 0 for packed interiors); only
 * interior cells are read or written.  Conserved-variable slot order is
 * HORMONE's (src/main/checksetup.f90:61-75): rho, m1, m2, m3, E, B1, B2,
 * B3, phi (the magnetic slots only with mag_on, phi only with mag_on and
 * dim > 1).
 */
#ifndef HORMONE_GPU_H
#define HORMONE_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HMN_OK 0
#define HMN_EINVAL (-1)     /* bad argument */
#define HMN_ENEG_EINT (-2)  /* negative internal energy: numflux.f90:579-593 / eos.f90:833-839 stop */
#define HMN_ECUDA (-3)      /* CUDA runtime error */
#define HMN_EBADCFG (-4)    /* configuration outside this path (checksetup.f90 stop) */
#define HMN_ENOMEM (-5)     /* device allocation failed */
#define HMN_ETIMEOUT (-6)   /* a bounded device wait ran out */

typedef struct hmn_ctx hmn_ctx;

/* Grid: the resolved indices and 1-D coordinate arrays of module `grid`
 * (src/main/modules.f90; filled by gridset.f90:40-140).  Each coordinate
 * array covers Fortran indices is-2..ie+2 (n+4 values). */
typedef struct {
  int n[3];           /* ie-is+1, je-js+1, ke-ks+1 */
  int ghost;          /* ghost layers of the caller's 3-D arrays (0 or 2) */
  int bc[3][2][2];    /* boundary codes [axis][inner,outer][scalar,vector], after checksetup.f90:109-128:
                       0 periodic, 1 reflective, 2 outgoing, 3 free, 4/5 linear, 9 Dirichlet,
                       10 flux (inner x3 face only) */
  const double* x[3];
  const double* xi[3];
  const double* dx[3];
  const double* dxi[3];
  const double* idx[3];
  const double* idxi[3];
} hmn_grid;

/* Settings of module `settings`/`physval`/`gravmod` used by the step. */
typedef struct {
  double gamma, courant, alpha9wave;
  double HGfac, hgcfl, alphagrv, G;
  int rktype;      /* 1, 2 or 3 */
  int grktype;     /* RK order of the gravity sub-steps */
  int limiter;     /* 0 flat, 1 minmod, 2 modified_mc */
  int mag_on;
  int gravswitch;  /* 0 off, 3 hyperbolic */
  int maxtngrv;
  int outstyle, endstyle;
  int precision;   /* 0 FP64 (bit-compatible), 1 FP32 flux / FP64 accumulation */
  int nspc;        /* passive scalars: spn with compswitch 2, else 0 (at most 8; FP64 single grids) */
} hmn_params;

/* allocations.f90 + metric.f90 for this grid: allocates device state. */
int hmn_create(const hmn_grid* grid, const hmn_params* params, hmn_ctx** out);

/* metric (src/main/metric.f90:102-151) for spherical polar coordinates
 * (crdnt 2: axes 1-3 are r, theta, phi, built as gridset.f90:294-423): the
 * 1-D factors module `grid` holds after `metric`, each from index is-2
 * (r) or js-2 (theta) to ie+2 / je+2.  sinc (sin of the arithmetic theta
 * centres) and sisin are read only with self-gravity (gravswitch 3). */
typedef struct {
  const double* detg1;   /* xi1**2 */
  const double* idetg1;
  const double* sx1;
  const double* sini;    /* sin and cos of the theta faces */
  const double* cosi;
  const double* scot;
  const double* sinc;
  const double* sisin;
} hmn_metric;

/* Sets the coordinate system; crdnt 0 (Cartesian, the default) takes no
 * arrays, crdnt 1 (cylindrical R, phi, z; metric.f90:53-100) only detg1,
 * idetg1 and sx1, and needs one phi cell (gridset.f90:209-231 reads an
 * unset width for the ghosts of a solved phi axis) and no gravity.  The kernels form idetg2, idetg3, dvol and sa1..3 from the 1-D
 * factors in the reference's operation order, and with gravswitch 3 the
 * spherical Laplacian coefficients of setup_grv_hyperbolic
 * (gravity_hyperbolic.f90:336-405; (r, theta) with one phi cell, or 3-D;
 * Robin outer radius, gbtype 1).  Spherical grids run as single grids in
 * either precision with r solved and without passive scalars (HMN_EBADCFG
 * otherwise).  Call before the first step. */
int hmn_set_metric(hmn_ctx* ctx, int crdnt, const hmn_metric* m);

/* Device copy of the state after initialcondition/conserve/pressure
 * (hormone.f90:94-100).  u: conserved array (ufnmax planes); prim: d, v1,
 * v2, v3, e, b1, b2, b3, phi as the reference holds them (NULL entries are
 * zero); grvphi/grvpsi: potential and its time derivative (may be NULL).
 * Any pointer may be NULL to leave that part unchanged. */
int hmn_upload(hmn_ctx* ctx, const double* u, const double* const prim[9], const double* grvphi,
               const double* grvpsi);

/* timestep (src/main/timestep.f90:15-105): CFL reduction on the device,
 * output/end clamps, ch = cfmax, and for gravswitch 3 cgrav and dtgrav.
 * Writes dt and ch (either pointer may be NULL). */
int hmn_timestep(hmn_ctx* ctx, double time, double t_out, double t_end, double* dt, double* ch);

/* gravity (src/main/gravity.f90:18-64 -> gravity_hyperbolic.f90:19-50):
 * the hyperbolic sub-cycles from grvtime to time+dt; tn is the step index
 * (tn == 0 only sets the boundary images, grav_init_other).  Refused
 * (HMN_EBADCFG) on a slab with gravity halos, which runs the sub-stages one
 * by one (below). */
int hmn_gravity_step(hmn_ctx* ctx, double time, double dt, int tn);

/* The same split into its sub-stages (for slabs, which exchange the
 * potential between them): hmn_gravity_begin plans the sub-cycles of
 * [time, time+dt] from the last dt/cgrav/dtgrav and writes *nsub =
 * tngrav x grktype (gravity_hyperbolic.f90:33-38; 0 at tn == 0, where only
 * the clock is set); hmn_gravity_substage runs the next RK sub-stage
 * (hyperbolic_gravity_step, gravity_hyperbolic.f90:62-110) and advances the
 * gravity clock after the last sub-stage of a cycle. */
int hmn_gravity_begin(hmn_ctx* ctx, double time, double dt, int tn, int* nsub);
int hmn_gravity_substage(hmn_ctx* ctx);

/* hydro_step (src/main/hydro.f90:15-52): rktype fused RK stages (boundary
 * images, slopes, HLLD fluxes, source, update, primitive check) with the dt
 * of the last hmn_timestep. */
int hmn_hydro_step(hmn_ctx* ctx);

/* phidamp (src/main/source.f90:239-260). */
int hmn_phidamp(hmn_ctx* ctx);

/* Host copy of the current state (output, restart dumps, the test harness,
 * tests.f90:46): u, the primitives d, v1, v2, v3, e, b1, b2, b3, phi as
 * rungekutta.f90:205-229 and phidamp leave them, and the potential.  NULL
 * pointers are skipped. */
int hmn_download(hmn_ctx* ctx, double* u, double* const prim[9], double* grvphi, double* grvpsi);

/* Boundary code 9 (Dirichlet, boundarycondition.f90:104-115,196-212): the
 * ghost values of face (axis 0-2, side 0 inner / 1 outer), i.e. the d0, p0,
 * v10, v20, v30, b10, b20, b30 (and spc0) of module physval there: 8 + nspc
 * planes, each 2 layers x the face's cells (layer l is the ghost at
 * coordinate -2+l on the inner side, n+l on the outer side; the other two
 * axes in increasing order, the lower one fastest).  Call again whenever
 * the values change.  Codes 4 and 5 (linear extrapolation, and linear with
 * outflow-only normal velocity) need no data; code 10 (the wind-tunnel flux
 * boundary, fluxboundary.f90) is not on this path. */
int hmn_set_dirichlet(hmn_ctx* ctx, int axis, int side, const double* vals);

/* Boundary code 10 (src/main/fluxboundary.f90:42-87, the wind-tunnel
 * inflow): the flux through the inner x3 face, replacing the Riemann flux
 * there after numflux (numflux.f90:566).  flux holds the 9 conserved slots
 * (d, m1, m2, m3, E, B1, B2, B3, phi) and then nspc scalar fluxes.  Only
 * axis 2, side 0, with bc3is = bc3iv = 10; the ghost layers beyond that
 * face, which the reference never rewrites, are set with hmn_set_dirichlet
 * as for code 9.  Both are needed before the first step. */
int hmn_set_flux_boundary(hmn_ctx* ctx, int axis, int side, const double* flux);

/* Passive scalars (compswitch 2: module physval's spc(1:spn,i,j,k), species
 * fastest, then i, j, k with the grid's ghost layers): upload the mass
 * fractions of the initial or restart state, or copy the current ones back.
 * They are advected with the mass flux as src/main/numflux.f90:200-212 and
 * rungekutta.f90:61-86 do. */
int hmn_upload_scalars(hmn_ctx* ctx, const double* spc);
int hmn_download_scalars(hmn_ctx* ctx, double* spc);

/* Gas pressure p = (gamma-1)*eint of the current state (eos.f90:742-794). */
int hmn_download_pressure(hmn_ctx* ctx, double* p);

/* Clock of the hyperbolic solver: grvtime and cgrav_old of module gravmod
 * (restored from a dump by readbin.f90:60-65). */
int hmn_set_gravity_clock(hmn_ctx* ctx, double grvtime, double cgrav_old);

/* Read the hyperbolic solver's clock (grvtime, cgrav_old), e.g. for the
 * cgrav_old record of a dump (output.f90:697-795).  Either pointer may be
 * NULL. */
int hmn_gravity_clock(hmn_ctx* ctx, double* grvtime, double* cgrav_old);

/* Asynchronous checkpoint of the current state: the data that write_bin
 * (src/main/output.f90:697-795) dumps for output and restart (d, v1, v2,
 * v3, e, b1, b2, b3, phi; grvphi and grvpsi with gravswitch 3), plus, when u
 * is not NULL, the conserved planes for an exact resume.  begin snapshots
 * the state on the device, ordered after the work enqueued so far, and
 * copies it to host staging on a separate stream while later steps run
 * (spc, if not NULL, receives the passive scalars as hmn_download_scalars);
 * wait blocks until that copy is done and fills the caller's arrays (laid
 * out as for hmn_download).  The arrays given to begin must stay valid until
 * wait returns.  One checkpoint is in flight at a time: begin first waits
 * for the previous one. */
int hmn_checkpoint_begin(hmn_ctx* ctx, double* u, double* const prim[9], double* grvphi, double* grvpsi,
                         double* spc);
int hmn_checkpoint_wait(hmn_ctx* ctx);

/* ---- slab decomposition along z -------------------------------------
 * One grid split into slabs of whole x-y planes, one per context (one per
 * GPU), as the reference's MPI domain decomposition (mpi_domain.F90:256-339,
 * timestep.f90:56,87) splits it across processes.  Each context is created
 * with its own slab: n[2] = the slab's layers (at least 2), the z coordinate
 * arrays of the slab (with 2 ghost entries each side), and any boundary
 * codes (those of an internal face are ignored).  hmn_set_slab hands it
 * four device buffers of hmn_slab_halo_bytes each, owned by the caller:
 * send_lo/send_hi receive the slab's two lowest/highest layers of every
 * primitive plane (hmn_pack_halos), recv_lo/recv_hi must hold the lower /
 * upper neighbour's send_hi / send_lo before each stage.  NULL recv/send
 * pointers mark a physical face (boundary codes apply).  wrap_lo/wrap_hi = 1
 * mark a face that is the grid's periodic z boundary (the first slab's low
 * face, the last slab's high face): its ghosts are formed as the periodic
 * boundary condition forms them (boundarycondition.f90:222-243 rebuilds
 * their energies from the pressure).  A step is then:
 *   hmn_cfl_local; all-reduce *min_dti (MIN) and *cfmax (MAX) from
 *   hmn_cfl_partials over the slabs (two doubles in device memory, ordered
 *   on hmn_stream); hmn_cfl_finalize -> dt, ch;
 *   for each RK stage s: hmn_pack_halos; exchange; hmn_hydro_stage(s);
 *   hmn_phidamp.
 * hmn_timestep, hmn_hydro_step and hmn_run refuse a context with
 * neighbours (HMN_EBADCFG). */
size_t hmn_slab_halo_bytes(const hmn_ctx* ctx);
int hmn_set_slab(hmn_ctx* ctx, double* send_lo, double* send_hi, const double* recv_lo, const double* recv_hi,
                 int wrap_lo, int wrap_hi);

/* Slabs of a 3-D Cartesian grid with hyperbolic self-gravity (gravswitch 3)
 * also exchange one layer of the potential: after hmn_set_slab, hand the
 * context four more buffers of hmn_slab_gravity_halo_bytes (NULL on the
 * same physical faces).  hmn_pack_gravity_halos copies the potential's
 * lowest / highest layer into send_lo / send_hi; recv_lo / recv_hi must hold
 * the lower / upper neighbour's send_hi / send_lo.  dtg_unit (the minimum
 * over all cells, tools.f90:160-183) must be the grid's: set every slab's to
 * the minimum of hmn_gravity_unit over the slabs.  A step is then
 *   hmn_cfl_local; all-reduce; hmn_cfl_finalize;
 *   hmn_gravity_begin(.., &nsub); nsub x { hmn_pack_gravity_halos;
 *   exchange; hmn_gravity_substage }; hmn_pack_gravity_halos; exchange;
 *   for each RK stage s: hmn_pack_halos; exchange; hmn_hydro_stage(s).
 * hmn_hydro_stage and hmn_gravity_begin refuse a gravity slab without them. */
size_t hmn_slab_gravity_halo_bytes(const hmn_ctx* ctx);
int hmn_set_slab_gravity(hmn_ctx* ctx, double* send_lo, double* send_hi, const double* recv_lo,
                         const double* recv_hi);
int hmn_pack_gravity_halos(hmn_ctx* ctx);
int hmn_gravity_unit(hmn_ctx* ctx, double* dtg_unit);
int hmn_set_gravity_unit(hmn_ctx* ctx, double dtg_unit);

/* The push exchange (instead of hmn_set_slab): recv_lo/recv_hi are this
 * slab's halo buffers (hmn_slab_halo_bytes each) for stage parity 0 and 1,
 * push_lo/push_hi the low and high neighbours' buffers that receive this
 * slab's bottom and top layers (the low neighbour's recv_hi, the high
 * neighbour's recv_lo; NULL entries on a physical face).  Each stage's
 * kernel stores its two boundary layers straight into the neighbours'
 * buffers while it writes them, so no pack kernel or message runs between
 * stages; on several GPUs the push buffers are the neighbours' memory
 * (peer access or symmetric memory).  Every slab must have finished a
 * stage before any starts the next (the caller's barrier).  Before the
 * first stage, and after any upload, hmn_pack_halos stores the current
 * layers.  3-D Cartesian grids without gravity. */
int hmn_set_slab_push(hmn_ctx* ctx, const double* const recv_lo[2], const double* const recv_hi[2],
                      double* const push_lo[2], double* const push_hi[2], int wrap_lo, int wrap_hi);

int hmn_pack_halos(hmn_ctx* ctx);
int hmn_hydro_stage(hmn_ctx* ctx, int stage);
int hmn_cfl_local(hmn_ctx* ctx, double time, double t_out, double t_end);
int hmn_cfl_partials(hmn_ctx* ctx, double** min_dti, double** cfmax);
int hmn_cfl_finalize(hmn_ctx* ctx, double* dt, double* ch);

/* Advance whole steps on the device without host round trips: the loop of
 * hormone.f90:126-155 (timestep, gravity, hydro_step, phidamp, time += dt)
 * until time >= t_end or max_steps steps; the clamps use t_out = t_end.
 * *time and *steps are updated. */
int hmn_run(hmn_ctx* ctx, double* time, double t_end, int max_steps, int* steps);

/* evo_output (src/main/output.f90:147-275): the totals of the current state
 * over the grid, out[0..9] = Mtot, Etot, Eitot, Ektot, Egtot, Mbound,
 * Ebound, Jbound, Ebtot, Jtot (the gravity entries with gravswitch 3,
 * Jbound/Jtot on cylindrical and spherical grids, else 0).  Summed per
 * block and then over blocks in a fixed order: deterministic, but not the
 * reference's sequential order.  The eq_sym doubling is the caller's. */
int hmn_evo(hmn_ctx* ctx, double out[10]);

/* First error recorded by any kernel: code and the cell (0-based). */
int hmn_last_error(hmn_ctx* ctx, int* code, int* i, int* j, int* k, int* sim);

/* Number of kernel launches issued by this context so far (diagnostics). */
long long hmn_launch_count(hmn_ctx* ctx);

/* Wait for all work of the context. */
int hmn_sync(hmn_ctx* ctx);

/* The context's CUDA stream (cudaStream_t), for callers that order their
 * own work after the step. */
void* hmn_stream(hmn_ctx* ctx);

int hmn_destroy(hmn_ctx* ctx);

/* ---- batches of independent simulations -------------------------------
 * Not in the reference (it advances one grid per process).  A batch holds
 * many simulations of uneven sizes in one device pool and advances all of
 * them, each on its own clock (its own CFL dt, t_end, ch), with one
 * persistent launch per phase; each simulation's result is bit-identical
 * to running it alone through hmn_create/hmn_run.  Supported grids: 3-D,
 * 2-D in the x-y plane and 1-D along x, boundary codes 0-5, no gravity,
 * one rktype per batch. */
typedef struct hmn_batch hmn_batch;

/* Device bytes one simulation of this grid occupies in a batch pool. */
size_t hmn_batch_footprint(const hmn_grid* grid, const hmn_params* params);

int hmn_batch_create(size_t pool_bytes, int max_sims, int precision, int rktype, hmn_batch** out);

/* Admit a simulation (state as for hmn_upload, packed layout, ghost = 0)
 * that runs from `time` to `t_end`; returns HMN_ENOMEM when the pool or the
 * slot table is full (the caller keeps it queued).  *sim = slot id. */
int hmn_batch_add(hmn_batch* b, const hmn_grid* grid, const hmn_params* params, const double* u,
                  const double* const prim[9], double time, double t_end, int* sim);

/* Release a simulation's slot and pool memory. */
int hmn_batch_remove(hmn_batch* b, int sim);

/* Advance every admitted, unfinished simulation that is not held by up to
 * nsteps steps (a simulation stops at its t_end).  Asynchronous. */
int hmn_batch_step(hmn_batch* b, int nsteps);

/* held[s] != 0 (one int per slot, max_sims of them) leaves simulation s out
 * of the following steps: its clock and state stay as they are until a
 * later call releases it (held[s] = 0).  A scheduler uses it to advance
 * small simulations alone between full steps; each simulation still takes
 * exactly its own sequence of steps.  No reference counterpart (the
 * reference runs one simulation per process). */
int hmn_batch_set_held(hmn_batch* b, const int* held);

/* Clock, step count, done flag and error code of every slot (arrays of
 * max_sims entries; any may be NULL).  Synchronises. */
int hmn_batch_poll(hmn_batch* b, double* time, int* tn, int* done, int* err);

/* Host copy of one simulation's state (u and the 9 primitive planes);
 * returns the simulation's error code (0 if none). */
int hmn_batch_download(hmn_batch* b, int sim, double* u, double* const prim[9]);

/* Schedule of one grid kind (0: 3-D, 1: 2-D x-y, 2: 1-D x): its tile
 * (tile_id 0 = 8x8x8 or 1 = 8x8x4 for 3-D, 2 = 16x16 or 3 = 32x8 for
 * 2-D, 4 = 256 for 1-D) and the persistent-grid size of the stage
 * launches in CTAs per SM (0: the occupancy limit).  The autotuner sets
 * it; results do not depend on it. */
int hmn_batch_set_schedule(hmn_batch* b, int kind, int tile_id, int blocks_per_sm);

/* Sweep schedule of one grid kind's stage launches: the order of the
 * (simulation, tile) work list and how the persistent CTAs split it.
 *   HMN_SWEEP_STATIC       simulations in slot order, each one's tiles x
 *                          fastest; CTA b takes items b, b + grid, ...
 *   HMN_SWEEP_INTERLEAVED  tile t of every simulation, then tile t + 1;
 *                          static split
 *   HMN_SWEEP_DYNAMIC      the largest simulations first; CTAs take the
 *                          next item from a shared counter
 * The autotuner sets it; results do not depend on it. */
#define HMN_SWEEP_STATIC 0
#define HMN_SWEEP_INTERLEAVED 1
#define HMN_SWEEP_DYNAMIC 2
int hmn_batch_set_sweep(hmn_batch* b, int kind, int sweep);

long long hmn_batch_launch_count(hmn_batch* b);
int hmn_batch_sync(hmn_batch* b);
void* hmn_batch_stream(hmn_batch* b);
int hmn_batch_destroy(hmn_batch* b);

/* The CFL timestep of hmn_timestep for callers that cannot allocate device
 * memory (no counterpart in the reference: HORMONE has no device code).
 * It needs no hmn_ctx: u_dev holds the conserved planes on the device
 * (packed interior, x fastest, ufnmax planes), and on completion out_dev
 * (3 doubles of caller-owned device memory) holds dt, ch and a status
 * (0, or HMN_ENEG_EINT if a cell has eint <= 0).  Work is enqueued on
 * `stream` (a cudaStream_t, NULL for the default stream); nothing is
 * synchronised.  The scratch is a static device array of 114,784 bytes
 * per GPU that loads the library: at most 4096 cells per axis (larger
 * grids return HMN_EINVAL), gravswitch must be 0, and the grid is taken
 * as Cartesian (a curvilinear grid's timestep goes through hmn_timestep,
 * which has its metric).  u_dev must be packed: grid->ghost other than 0
 * returns HMN_EINVAL.  The first call on a device allocates: the CUDA
 * runtime loads the library's device code there (and with it the array)
 * and the call looks up the array's address, so make it at start-up.
 * Every call copies grid->dxi from host memory on `stream`, so it must not
 * be called while that stream is being captured into a CUDA graph.  Calls
 * that overlap on the GPU share the array and race: the caller must order
 * them. */
int hmn_timestep_noalloc(const hmn_grid* grid, const hmn_params* params, const double* u_dev, double time,
                         double t_out, double t_end, double* out_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif
