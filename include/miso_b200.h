/*
 * miso_b200.h -- C ABI of libmiso_b200.so, the B200 (sm_100a) implementation
 * of MISO's explicit ideal-MHD time step.
 *
 * Every call returns an int status (MISO_B200_OK = 0, negative on error) and
 * never aborts the process; miso_b200_last_error() gives a message.  One
 * handle is driven by one host thread; all device work of a handle is
 * ordered on one CUDA stream (the caller's, or one the handle creates).
 *
 * Field order everywhere: ro, vx, vy, vz, bx, by, bz, ei, ph -- the
 * reference's primitive variables (miso/include/miso/mhd_fields.hpp:17-18),
 * each an (i_total, j_total, k_total) array with k fastest
 * (miso/include/miso/array3d.hpp:54-60) and `margin` ghost cells on every
 * axis of size > 1 (miso/include/miso/grid.hpp:67-90).
 */
#ifndef MISO_B200_H
#define MISO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MISO_B200_OK 0
#define MISO_B200_ERR_ARG (-1)      /* invalid argument or descriptor */
#define MISO_B200_ERR_CUDA (-2)     /* a CUDA call failed */
#define MISO_B200_ERR_NONFINITE (-3) /* non-positive/non-finite ro or ei seen by the CFL pass */
#define MISO_B200_ERR_STATE (-4)    /* call not valid in the handle's current state */
#define MISO_B200_ERR_NOMEM (-5)    /* device allocation failed */
#define MISO_B200_ERR_TIMEOUT (-6)  /* a bounded device-side wait (TMA copy) ran out */
#define MISO_B200_ERR_HALO (-7)     /* the halo exchange callback reported an error */
#define MISO_B200_ERR_CALLBACK (-8) /* the boundary callback reported an error */

#define MISO_B200_FP64 0        /* primitive FP64 state, bit-faithful to the reference */
#define MISO_B200_FP32_SPLIT 1  /* conserved FP32 hi/lo state, FP32 RHS and viscosity */

/* Grid and boundary description.  Replaces the serial constructor
 * Grid<Real, backend::Host>(i_size, ..., z_max) (miso/include/miso/grid.hpp:316-337),
 * domain.periodic.{x,y,z} (miso/include/miso/mpi_util.hpp:79-86) and the
 * demos' symmetric "outflow" boundary functor
 * (demo/mhd1d_shock_tube/src/main.cpp:85-162 calling
 * boundary_condition::symmetric, miso/include/miso/boundary_condition.hpp:109-136). */
typedef struct miso_b200_grid_desc {
  int i_size, j_size, k_size; /* interior cells per axis (size 1 = degenerate axis) */
  int margin;                 /* ghost width on non-degenerate axes; the stencil needs 2 */
  double x_min, x_max, y_min, y_max, z_min, z_max;
  int periodic[3];            /* 1 = periodic wrap; 0 = mirror (symmetric) faces */
  double sign[3][2][9];       /* mirror sign per axis, side (0 inner, 1 outer), field */
} miso_b200_grid_desc;

/* Physics and numerics parameters: the keys the reference's integrator reads
 * (eos.gm, eos.hpp:17; mhd.cfl_number, mhd_integrator_host.hpp:52;
 * mhd.artificial_viscosity.*, mhd_artificial_viscosity_host.hpp:40-44). */
typedef struct miso_b200_params {
  double gm;
  double cfl_number;
  double ep, fh;
  double cs_fac, ca_fac, vv_fac;
  int precision; /* MISO_B200_FP64 or MISO_B200_FP32_SPLIT */
} miso_b200_params;

typedef struct miso_b200_handle miso_b200_handle;

/* Create a solver for one grid on the current CUDA device.  `stream` is a
 * cudaStream_t (NULL: the handle creates its own).  Replaces the
 * construction of Integrator<Real, backend::CUDA> with its workspaces
 * (miso/include/miso/mhd_integrator_cuda.cuh:328-339) and of Fields qq
 * (miso/include/miso/mhd.hpp:22-25). */
int miso_b200_create(const miso_b200_grid_desc *grid, const miso_b200_params *params,
                     void *stream, miso_b200_handle **out);

/* Release every device buffer of the handle. */
int miso_b200_destroy(miso_b200_handle *h);

/* Copy the 9 primitive fields in (q[f] host or device pointers, full arrays
 * including ghosts).  Replaces Fields<Real, CUDA>::copy_from(host Fields)
 * (miso/include/miso/mhd_fields.hpp:150-160).  Synchronises the stream. */
int miso_b200_upload(miso_b200_handle *h, const double *const q[9]);

/* Copy the 9 primitive fields out (FP32_SPLIT: converted from the conserved
 * hi/lo state to FP64 primitives).  Replaces Fields<Real, Host>::copy_from(CUDA
 * Fields) (miso/include/miso/mhd_fields.hpp:83-96).  Synchronises the stream. */
int miso_b200_download(miso_b200_handle *h, double *const q[9]);

/* miso_b200_download without waiting: the conversion and the copies are
 * enqueued on the handle's stream and `event` (a cudaEvent_t created by the
 * caller, or NULL) is recorded after the last copy; q[] must stay valid
 * (and, for overlap with host work, be pinned) until the event completes.
 * Steps enqueued afterwards are ordered after the copies, so a snapshot can
 * drain while the simulation goes on.  No counterpart in the reference,
 * whose Checkpoint::save copies synchronously (mhd_checkpoint.hpp:35-62). */
int miso_b200_download_async(miso_b200_handle *h, double *const q[9], void *event);

/* Fill every ghost cell from its periodic or mirror image.  Replaces
 * Integrator::apply_boundary_condition(bc, qq) for the built-in boundaries
 * (miso/include/miso/mhd_integrator_cuda.cuh:396-401). */
int miso_b200_fill_ghosts(miso_b200_handle *h);

/* CFL time step, returned to the host (synchronises).  Replaces
 * Integrator::cfl(qq, eos) (miso/include/miso/mhd_integrator_cuda.cuh:450-478,
 * host twin mhd_integrator_host.hpp:303-334).  The result is also kept on
 * the device for miso_b200_update_device(). */
int miso_b200_cfl(miso_b200_handle *h, double *dt_out);

/* Advance one step with a host-given dt: 4 Runge-Kutta stages, 3 artificial
 * viscosity sweeps, ghost fills.  Replaces Integrator::update(dt, eos, bc,
 * src, qq) (miso/include/miso/mhd_integrator_cuda.cuh:481-487; host twin
 * mhd_integrator_host.hpp:344-350).  Asynchronous. */
int miso_b200_update(miso_b200_handle *h, double dt);

/* Advance one step with the dt left on the device by the last CFL pass
 * (no host round trip).  Asynchronous. */
int miso_b200_update_device(miso_b200_handle *h);

/* Run `nsteps` of ModelBase::update() -- cfl then update
 * (miso/include/miso/mhd_model_base.hpp:57-62) -- with dt kept on the device.
 * With use_graph != 0 one step is captured in a CUDA graph on first use and
 * replayed.  Asynchronous. */
int miso_b200_run(miso_b200_handle *h, int nsteps, int use_graph);

/* The time loop of ModelBase::run between two outputs, kept on the device
 * (mhd_model_base.hpp:108-111 with ModelBase::update, :57-62, and
 * Time::update, time.hpp:64-67): steps -- CFL, update, time += dt, dt kept
 * on the device as miso_b200_run does -- while time < t_end and fewer than
 * max_steps steps were taken, checked after every step as the reference's
 * loop checks it.  *time is the time before (in) and after (out); *steps
 * the steps taken.  With use_graph the loop is one CUDA graph launch: a
 * conditional WHILE node whose condition a one-thread kernel sets after
 * each step from the device-held time (where a step swaps the FP32-split
 * hi / lo sets the body holds two steps, the second under an IF node with
 * the same condition).  Without it, or with a boundary callback, the steps
 * are launched from the host and the time is read after each.
 * Synchronises.  ERR_STATE on a shard (its dt is reduced on the host). */
int miso_b200_run_until(miso_b200_handle *h, double *time, double t_end, int max_steps,
                        int use_graph, int *steps);

/* Wait for the handle's stream; reports device-side error flags. */
int miso_b200_sync(miso_b200_handle *h);

/* dt of the last CFL pass as held on the device (synchronises). */
int miso_b200_last_dt(miso_b200_handle *h, double *dt_out);

/* FP64 global monitors of the current state: out[0..7] = sum ro dV,
 * sum ro*vx dV, sum ro*vy dV, sum ro*vz dV, sum Et dV, sum |div B| dV,
 * max |div B|, sum ph^2 dV (interior cells, dV = product of the spacings of
 * the non-degenerate axes).  Synchronises. */
int miso_b200_monitors(miso_b200_handle *h, double out[8]);

/* Fold the monitors' sums into the step (3-D FP32-split grids; ERR_STATE
 * otherwise): with on != 0 the last viscosity sweep of every step also
 * leaves FP64 per-block sums of the new state's mass, momentum, energy and
 * ph^2, and miso_b200_monitors() then reduces only |div B| (a kernel that
 * reads bx, by, bz) instead of the whole state.  For loops that read the
 * monitors after every step.  Applies with the default z sweep (variant 0)
 * and with the fused y and z sweeps (y variant 3); the results equal the
 * unfused monitors up to FP64 summation order. */
int miso_b200_set_monitor_fusion(miso_b200_handle *h, int on);

/* Device pointers of the FP64 primitive state arrays (FP64 form only), valid
 * until the next call that steps or destroys the handle.  Gives user code
 * the reference's FieldsView for custom boundary work
 * (miso/include/miso/mhd_fields.hpp:17-34). */
int miso_b200_fields_view(miso_b200_handle *h, double *ptrs[9]);

/* Built-in source term of the momentum and energy equations: the Source
 * argument of Integrator::update (miso/include/miso/mhd_integrator_host.hpp:
 * 134-168 and 241; concept mhd_model_base.hpp:131-155), default
 * EmptySourceTerm.  MISO_B200_SOURCE_POINT_GRAVITY is the magnetosphere
 * demo's gravity (demo/mhd3d_magnetosphere/src/src.hpp:17-44): force per
 * volume -ro g x / |x|^3 about the coordinate origin, params[0] = g, no
 * heating.  Both forms: FP64 bit for bit as the reference adds it; in the
 * FP32 split form the force is formed in FP32 and the 3-D RK stage runs
 * variant 2 or 3 (set_variant of another RK variant is refused while a
 * source is on).  Every cell centre must lie off the origin. */
#define MISO_B200_SOURCE_NONE 0
#define MISO_B200_SOURCE_POINT_GRAVITY 1
int miso_b200_set_source(miso_b200_handle *h, int kind, const double *params, int nparams);

/* Boundary functor.  Replaces the `bc` argument of Integrator::update /
 * apply_boundary_condition (miso/include/miso/mhd_integrator_host.hpp:
 * 250-255) for a boundary other than the descriptor's per-face mirror /
 * periodic one.  MISO_B200_BOUNDARY_FACES (the default) is that one.
 * MISO_B200_BOUNDARY_MAGNETOSPHERE is the magnetosphere demo's boundary
 * (demo/mhd3d_magnetosphere/src/bc.hpp:39-158), applied after every pass as
 * the reference applies its functor:
 *   - the descriptor's mirror faces;
 *   - in the x-inner ghosts, ro, vx, ei and bz set to the solar wind
 *     (ei = pr_sw / (gm - 1) / ro_sw);
 *   - on every cell, ghosts included, each field blended toward the state
 *     of miso_b200_set_blend_state (zeros until set) with weight
 *     f = a0 h / (a0 h + 1), h = max(0, (r / radius)^2 - 1), r the distance
 *     from the coordinate origin;
 *   - floors ro >= ro_floor and ei >= pr_floor / (gm - 1) / ro.
 * The maxima are rounded through float, as the reference's util::max2 is.
 * params: [0] ro_sw, [1] pr_sw, [2] vx_sw, [3] bz_imf, [4] radius, [5] a0,
 * [6] ro_floor, [7] pr_floor, [8] nonzero: miso_b200_cfl masks the sphere
 * r <= radius as the demo's TimeStep::cfl does (timestep.hpp:15-49).
 * Non-periodic axes only (ERR_ARG otherwise).  The FP64 form stays bit for
 * bit the reference's.  The FP32 split form applies the same steps to the
 * primitives it forms in FP64 from its conserved state, after every pass,
 * and runs its per-cell kernels (which read every ghost cell) while the
 * boundary is on; on a grid decomposed into shards it is refused
 * (ERR_STATE). */
#define MISO_B200_BOUNDARY_FACES 0
#define MISO_B200_BOUNDARY_MAGNETOSPHERE 1
int miso_b200_set_boundary(miso_b200_handle *h, int kind, const double *params, int nparams);
/* The state the magnetosphere boundary blends toward: 9 primitive arrays
 * with ghosts, host or device pointers, copied.  The demo allocates this
 * state and never writes it; a caller passes the initial condition, or
 * zeros for the demo as it runs on zero-filled memory. */
int miso_b200_set_blend_state(miso_b200_handle *h, const double *const q[9]);

/* Mirror signs of the descriptor's non-periodic faces, set after create:
 * sign[(axis * 2 + side) * 9 + field], +1 or -1 (axis 0..2 = x, y, z; side
 * 0 inner, 1 outer), as boundary_condition::symmetric's Sign
 * (miso/include/miso/boundary_condition.hpp:109-136).  Ghosts keep their
 * values until the next fill (miso_b200_fill_ghosts or a step). */
int miso_b200_set_mirror_signs(miso_b200_handle *h, const double *sign);

/* A boundary functor of the caller's own, FP64 form: the `bc` argument of
 * Integrator::update / apply_boundary_condition for a boundary the built-in
 * faces do not describe.  After every pass -- where the reference calls
 * bc.apply(qq.view(), grid.const_view()) and then its halo exchange
 * (miso/include/miso/mhd_integrator_cuda.cuh:396-401, host twin
 * mhd_integrator_host.hpp:250-255) -- the library waits for its stream,
 * calls fn(user, q, stream) with the 9 primitive arrays of the state just
 * written (on_host != 0: host copies in pinned memory, copied back to the
 * device after the call; on_host == 0: the device arrays themselves), and
 * then fills the periodic faces.  The non-periodic faces are left to the
 * callback.  A nonzero return is reported as MISO_B200_ERR_CALLBACK.  This
 * is the slow path (a host round trip per pass, 7 per step, and no CUDA
 * graph: miso_b200_run with use_graph returns MISO_B200_ERR_STATE).
 * fn == NULL returns to the descriptor's faces.  ERR_STATE on the split
 * form, with a halo exchange or with the magnetosphere boundary. */
typedef int (*miso_b200_boundary_fn)(void *user, double *const q[9], void *stream);
int miso_b200_set_boundary_callback(miso_b200_handle *h, miso_b200_boundary_fn fn, void *user,
                                    int on_host);

/* Halo exchange of a grid decomposed into shards along i (the slowest
 * axis).  Replaces the reference's HaloExchanger for the neighbour faces of
 * a Cartesian decomposition (miso/include/miso/mhd_halo_exchange.hpp:
 * 451-621) and the MPI_Allreduce of dt in Integrator::cfl
 * (miso/include/miso/mhd_integrator_cuda.cuh:476).  A face's ghost layer
 * along i is `margin` whole planes of each array, contiguous in memory, so
 * nothing is packed: the callback moves `bytes` contiguous bytes per array
 * and face.
 *
 * exchange: called on the host whenever a pass has written arrays whose i
 *   ghosts the next pass reads.  It must make `stream` (the handle's
 *   cudaStream_t) wait until, for every array a and every face marked
 *   external, send_lo[a] has reached the low neighbour's recv_hi[a] and the
 *   low neighbour's send_hi[a] has reached recv_lo[a] (high face alike:
 *   send_hi[a] -> high neighbour's recv_lo[a], its send_lo[a] ->
 *   recv_hi[a]).  Typically: a group of ncclSend/ncclRecv on `stream`, or
 *   cudaMemcpyAsync between shards of one process.  Nonzero return =
 *   MISO_B200_ERR_HALO.  Arrays are double (FP64) or float (FP32 split).
 * min_all: minimum of *value over all shards, written back (host value);
 *   NULL = this shard alone.  miso_b200_cfl() returns the global dt with it.
 *
 * ext_lo / ext_hi mark the low / high i face as shared with a neighbour
 * (its ghosts come from the exchange, never from a periodic or mirror
 * image); a face not marked keeps the grid descriptor's boundary.  With
 * ops == NULL the handle returns to a single grid.  While halo exchange is
 * on, steps are taken with miso_b200_cfl + miso_b200_update (host dt, the
 * reference's own sequence); miso_b200_run and miso_b200_update_device
 * return MISO_B200_ERR_STATE.  miso_b200_monitors covers this shard only. */
typedef struct miso_b200_halo_ops {
  int (*exchange)(void *user, int narrays, size_t bytes, int ext_lo, int ext_hi,
                  void *const *send_lo, void *const *send_hi, void *const *recv_lo,
                  void *const *recv_hi, void *stream);
  int (*min_all)(void *user, double *value);
  void *user;
} miso_b200_halo_ops;

int miso_b200_set_halo(miso_b200_handle *h, int ext_lo, int ext_hi,
                       const miso_b200_halo_ops *ops);

/* Halo exchange of a grid decomposed along any of i, j and k: the
 * reference's full Cartesian decomposition (miso/include/miso/grid.hpp:
 * 279-313, one box per rank; HaloExchanger::apply exchanging the x, y and z
 * faces, mhd_halo_exchange.hpp:451-621).  ext[2 * axis + side] marks the
 * low (side 0) / high (side 1) face of axis 0, 1, 2 (i, j, k) as shared
 * with a neighbour.  The exchange callback takes the axis and is called
 * once per axis with a shared face, with the contract of
 * miso_b200_halo_ops.exchange above.  Along i the pointers are the arrays'
 * own planes; a j or k face is not contiguous, so the library gathers the
 * `margin` interior layers next to each shared face (the full extent of the
 * other two axes, ghosts included, in the arrays' memory order) into
 * buffers of its own before the call and scatters recv_lo / recv_hi into
 * the ghost layers after it, on `stream` (the reference's pack_y_send /
 * unpack_y_recv, mhd_halo_exchange.hpp:303-335, 395-424); `bytes` is one
 * array's face.  A pass is followed by the exchanges the next pass reads:
 * every axis after a Runge-Kutta stage and after the step's last viscosity
 * sweep, j after the x sweep, k after the y sweep.  With a shared k face the
 * y and z sweeps run as two passes (y sweep variant 3 runs as the line y
 * sweep and the z sweep the handle's z variant), and the overlapped
 * exchange is refused (it covers i faces only).  min_all, ops == NULL and
 * the stepping rules as for miso_b200_set_halo, which is this call with
 * ext = {ext_lo, ext_hi, 0, 0, 0, 0}. */
typedef struct miso_b200_halo3_ops {
  int (*exchange)(void *user, int axis, int narrays, size_t bytes, int ext_lo, int ext_hi,
                  void *const *send_lo, void *const *send_hi, void *const *recv_lo,
                  void *const *recv_hi, void *stream);
  int (*min_all)(void *user, double *value);
  void *user;
} miso_b200_halo3_ops;

int miso_b200_set_halo3(miso_b200_handle *h, const int ext[6], const miso_b200_halo3_ops *ops);

/* A source functor of the caller's own, for either form: the reference's
 * Source concept (src.vx, src.vy, src.vz, src.ei evaluated on the stage's
 * argument state, mhd_model_base.hpp:131-155), as update_sc4 uses it
 * (mhd_integrator_host.hpp:134, 151, 168: the forces inside the dt factor
 * of the momentum equations; 241: src.ei added to the new total energy
 * outside it).  Before every Runge-Kutta stage `fn` gets the stage's
 * argument state q[9] (primitive fields, ghosts included, the handle's
 * field layout) and fills s[0..3] (four arrays of the same layout) with the
 * four terms of every interior cell; it returns 0, or any other value to
 * stop the step with MISO_B200_ERR_CALLBACK.  on_host != 0: q and s are
 * host copies that the library stages (exact, and slow); 0: device arrays,
 * with the handle's stream as the last argument.  While set it replaces the
 * built-in source; fn == NULL removes it.  In the FP32 split form q holds the
 * stage's argument state converted to FP64 primitives (hi + lo words for the
 * step's first stage, the FP32 stage buffer otherwise), the terms enter the
 * FP32 right-hand side, and the last stage's update is not deferred into the
 * x sweep while a callback is set.  ERR_STATE on a grid in shards; no graph
 * capture
 * (miso_b200_run with use_graph refuses, miso_b200_run_until launches the
 * steps from the host). */
typedef int (*miso_b200_source_fn)(void *user, const double *const q[9], double *const s[4],
                                   void *stream);
int miso_b200_set_source_callback(miso_b200_handle *h, miso_b200_source_fn fn, void *user,
                                  int on_host);

/* Overlap each halo exchange with the pass after it (3-D FP32-split grids on
 * the pipelined Runge-Kutta stage and the line x sweep, the defaults;
 * ERR_STATE otherwise or without a halo exchange).  The exchange callback
 * is then called with `comm_stream` (a cudaStream_t of the caller's) as its
 * stream, ordered after the pass that wrote the planes; the next pass that
 * reads across i -- a Runge-Kutta stage or the x sweep -- first finishes the
 * planes [2, n-2), which read no ghost plane, then waits for the exchange
 * and finishes the two boundary groups [0, 2) and [n-2, n).  The results
 * are the same bits as without overlap.  Shards of one process on one GPU
 * share one comm stream, as they share one stream.  comm_stream == NULL
 * turns the overlap off.  No counterpart in the reference, whose halo
 * exchange blocks between passes (mhd_halo_exchange.hpp:451-621). */
int miso_b200_set_halo_overlap(miso_b200_handle *h, void *comm_stream);

/* Kernel variant of one kernel class on the 3-D FP32-split path:
 * kernel_class 0 = Runge-Kutta stage, 1/2/3 = viscosity sweep x/y/z;
 * variant 0 = tiled (TMA plane tiles / streaming lines fed by a producer
 * warp / warp-shuffle rows), 1 = flat (one thread per cell), 2 = pipelined
 * (Runge-Kutta stage: TMA planes with packed FP32x2 differences; x / y
 * sweeps: one warp per line segment marching along the sweep axis; z sweep:
 * k rows streamed by TMA), 3 (Runge-Kutta stage only, the default) = variant 2 with the last
 * stage's update deferred into the x sweep: that stage writes its
 * right-hand side and the x sweep forms the new state from it as it streams
 * the state in (this needs x sweep variant 0 and no flat sweep; otherwise
 * it runs as variant 2), and 3 (y sweep only) = the y and z sweeps fused
 * into one pass: each k column of a plane is swept along j and each finished
 * row along k, with the separate sweeps' arithmetic, so the step gives the
 * same bits as the y line sweep followed by the z sweep without writing
 * and re-reading the y-swept state (the z variant is then unused).  All
 * compute the same step up to FP32 rounding order; the
 * autotuner (miso_b200/autotune.py) times them and keeps the fastest.
 * ERR_STATE on grids that use the simple per-cell kernels only. */
int miso_b200_set_variant(miso_b200_handle *h, int kernel_class, int variant);
int miso_b200_get_variant(miso_b200_handle *h, int kernel_class, int *variant);

/* Planes per work item along the march axis for the Runge-Kutta and the
 * x/y viscosity kernels of the 3-D FP32-split path (defaults 64 and 128). */
int miso_b200_set_chunks(miso_b200_handle *h, int rk_chunk, int av_chunk);

/* Bound, in SM clock cycles, of the waits in which the consumer threads of
 * the 3-D FP32-split Runge-Kutta stage and x / y sweep kernels wait for
 * each plane's TMA copy (default, and cycles <= 0: 4e9, about 2 s).  A wait
 * that runs out sets the handle's timeout flag; the kernel waits (with the
 * default bound) for its copies still in flight and returns, and the next
 * synchronising call reports MISO_B200_ERR_TIMEOUT.  For tests of that
 * path: a bound far below a copy's latency makes every wait run out.  No
 * counterpart in the reference, whose CUDA errors abort the process
 * (miso/include/miso/cuda_util.cuh:17-33).  ERR_STATE on other grids. */
int miso_b200_set_wait_limit(miso_b200_handle *h, long long cycles);

/* A test of the timeout path without a fault: the next pipelined Runge-Kutta
 * stage launched outside a CUDA-graph capture (miso_b200_update,
 * miso_b200_update_device, miso_b200_run without a graph) first waits, with
 * bound `cycles`, on an mbarrier phase that nothing completes.  The wait
 * runs out; the kernel sets the timeout flag, waits for its copies in flight
 * and returns, and the next synchronising call reports
 * MISO_B200_ERR_TIMEOUT.  The step's state is then invalid; the context and
 * other handles are not affected.  One launch only.  ERR_STATE unless the
 * handle runs a 3-D split grid on the pipelined stage (variant 2 or 3). */
int miso_b200_arm_timeout_test(miso_b200_handle *h, long long cycles);

/* Enable (1) or disable (0) per-kernel CUDA-event timing on the handle's
 * stream (outside graph replays); clears the accumulated totals. */
int miso_b200_set_timing(miso_b200_handle *h, int enable);

/* Per-kernel totals since the last miso_b200_set_timing(), as JSON text
 * {"name": {"launches": n, "ms": total, "bytes": algorithmic bytes}, ...}.
 * Synchronises. */
int miso_b200_timing_report(miso_b200_handle *h, char *buf, size_t len);

/* Bytes of device memory the handle holds. */
int miso_b200_device_bytes(miso_b200_handle *h, size_t *bytes);

/* Number of kernels the library enqueued on the handle's stream so far. */
int miso_b200_launch_count(miso_b200_handle *h, long long *count);

/* ---------------------------------------------------------------------------
 * Batched solver: `count` independent grids (any mix of 1-D, 2-D and 3-D,
 * uneven sizes, their own parameters) advanced together.  Every pass of a
 * step is one persistent launch over a list of 256-cell tiles of all
 * instances; each instance keeps its own time step (per-instance CFL
 * minimum).  No counterpart in the reference, which runs one grid per
 * process (mhd_model_base.hpp:89-116); each instance follows the same
 * update as miso_b200_update.  All instances share params[0].precision.
 * ------------------------------------------------------------------------- */
typedef struct miso_b200_batch miso_b200_batch;

int miso_b200_batch_create(int count, const miso_b200_grid_desc *grids,
                           const miso_b200_params *params, void *stream,
                           miso_b200_batch **out);
int miso_b200_batch_destroy(miso_b200_batch *b);
/* Copy instance `index`'s 9 primitive fields in / out (host or device pointers). */
int miso_b200_batch_upload(miso_b200_batch *b, int index, const double *const q[9]);
int miso_b200_batch_download(miso_b200_batch *b, int index, double *const q[9]);
/* Fill every instance's ghost cells from their images. */
int miso_b200_batch_fill_ghosts(miso_b200_batch *b);
/* nsteps of (per-instance cfl, update); with use_graph a step is captured
 * once and replayed.  Asynchronous. */
int miso_b200_batch_run(miso_b200_batch *b, int nsteps, int use_graph);
/* Wait for the batch's stream; reports device-side error flags. */
int miso_b200_batch_sync(miso_b200_batch *b);
/* Time step of each instance's last step (count values; synchronises). */
int miso_b200_batch_dt(miso_b200_batch *b, double *dt);
/* Interior cells of all instances, tiles in the work list, kernels enqueued. */
int miso_b200_batch_info(miso_b200_batch *b, long long *interior_cells, int *tiles,
                         long long *launches);
/* Planes per work item of the 3-D instances' Runge-Kutta stage and x / y
 * sweeps (as miso_b200_set_chunks; defaults 64 and 128).  3-D FP32-split
 * instances that take the tiled path run the single grid's pipelined
 * kernels, each instance on its own stream forked from the batch's stream
 * every step; short work items keep more of them in flight at once.  The
 * autotuner (miso_b200/autotune.py, autotune_batch) picks these per batch
 * composition. */
int miso_b200_batch_set_chunks(miso_b200_batch *b, int rk_chunk, int av_chunk);
/* Kernel variant (as miso_b200_set_variant) of the 3-D instances that run
 * the pipelined kernels; the autotuner tries the warp-march x / y sweeps,
 * which suit grids narrower than the line sweeps' 128-cell k blocks. */
int miso_b200_batch_set_variant(miso_b200_batch *b, int kernel_class, int variant);
/* Number of instances the batch runs through the pipelined kernels. */
int miso_b200_batch_views(miso_b200_batch *b, int *views);
const char *miso_b200_batch_last_error(miso_b200_batch *b);

/* Allocation-free CFL time step.  No counterpart in the reference: it is an
 * extra entry point for callers that cannot let a library allocate device
 * memory -- applications that give every byte of device memory to their
 * own pool or hold it to a fixed budget, and applications whose other
 * streams must not be stalled by the device-wide synchronisation that
 * cudaMalloc / cudaFree can cause.  It computes the same float-rounded CFL
 * time step as miso_b200_cfl() over the interior of 9 caller-owned DEVICE
 * arrays q[] (FP64 primitives ro, vx, vy, vz, bx, by, bz, ei, ph in the
 * layout above, ghosts included) and returns it in *dt_out (host), with no
 * handle and no cudaMalloc/cudaFree: its scratch is a 65,792-byte array in
 * the library's device memory, held by every GPU that loads the library
 * until the process exits.  Grids of more than 268,435,456 interior cells
 * are rejected with MISO_B200_ERR_ARG, and so are pointers that are not
 * device memory of the current device or arrays shorter than the grid
 * (checked before any launch, with queries that allocate nothing).  The
 * first call on a device looks up that device's scratch address.  Every
 * call shares the one scratch array: calls whose work overlaps on the GPU
 * (other threads, other streams) race and must be serialised by the
 * caller.  The call copies the result to the host and waits for `stream`
 * (a cudaStream_t, NULL = default stream) before it returns. */
int miso_b200_cfl_noalloc(const miso_b200_grid_desc *grid, const miso_b200_params *params,
                          const double *const q[9], void *stream, double *dt_out);

/* Message of the last error on this handle (or, when h is NULL, of the last
 * failed create or miso_b200_cfl_noalloc call). */
const char *miso_b200_last_error(miso_b200_handle *h);

/* Where a pointer lives: *kind = 1 for device (or managed) memory of any
 * GPU, 0 for host memory (pageable or pinned).  Allocates nothing. */
int miso_b200_pointer_kind(const void *p, int *kind);

/* Memory that host code and device code can both read and write (CUDA
 * managed memory), for data a device functor of the caller's reads -- the
 * C++ backend keeps the grid's coordinate arrays there, so a source functor
 * holding a view of the grid runs on either side.  *ptr = NULL for bytes ==
 * 0; MISO_B200_ERR_NOMEM when the allocation fails (no GPU, or out of
 * memory).  miso_b200_free_shared releases such a block (NULL: no-op). */
int miso_b200_alloc_shared(size_t bytes, void **ptr);
int miso_b200_free_shared(void *ptr);

/* Library version string. */
const char *miso_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif
