/* cdns.h -- C ABI of the B200 (sm_100a) channel-dns time step.
 *
 * This library replaces the per-time-step hot path of the reference solver
 * (hesse-x/channel-dns): the body of Simulation::enqueue_serial_step
 * (src/sim/simulation.cpp:142-171) together with the objects it drives --
 * Transforms::xyzfft2_impl (src/fft/transforms.cpp:615-741),
 * vector_ops::enqueue_curl / enqueue_cross_product
 * (src/solver/vector_ops.cpp:112-151, :250-272), TimeStepper
 * (src/solver/timestepper.cpp:19-68), EqSolvePV::setup / solve_modes
 * (src/solver/eqsolve_pv.cpp:311-509) and Simulation::correct_flow
 * (src/sim/simulation.cpp:111-140).  The reference's C++ driver keeps config
 * parsing, restart/physical output and statistics; it hands the state over
 * in its own memory layout.
 *
 * Conventions
 *  - Every function returns CDNS_OK (0) or a nonzero cdns_status; no C++
 *    exception crosses the ABI and device code never traps.  The message of
 *    the last failure on the calling thread is available from
 *    cdns_last_error().
 *  - Complex arrays are interleaved (re, im) doubles in the reference layout
 *    (src/core/array4d.hpp:62-67, src/solver/fields.hpp:17-22):
 *      velocity   [2*NZS+1][NYS+1][NXS+1][3]   (component innermost)
 *      pressure   [2*NZS+1][NYS+1][NXS+1]
 *      vel. BC    [2*NZS+1][2][NXS+1][3]       (wall 0 is y=+1, wall 1 is y=-1)
 *      fine phys. [NZ2][NY2+1][NX2]            (real)
 *    Host pointers may be pageable or pinned; *_device variants take device
 *    pointers on the context's GPU and copy on the context's stream.
 *  - One context per host thread; the context owns its CUDA stream, its
 *    device buffers and its captured step graphs.
 */
#ifndef CDNS_H
#define CDNS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CDNS_OK = 0,
    CDNS_ERR_ARG = 1,         /* bad argument, size or unsupported mesh */
    CDNS_ERR_CUDA = 2,        /* CUDA runtime failure */
    CDNS_ERR_STATE = 3,       /* call out of order (e.g. step before set_velocity) */
    CDNS_ERR_NONFINITE = 4,   /* the step produced NaN/Inf (reference: finite check) */
    CDNS_ERR_PIVOT = 5,       /* zero or non-finite tau pivot / flow response */
    CDNS_ERR_NOMEM = 6        /* device allocation failed */
} cdns_status;

/* Arithmetic of the step.  FP64: everything in double (the drop-in).  MIXED:
 * the fine-grid stage buffers and the z/x FFTs and products u x omega are
 * FP32 (the y synthesis/analysis accumulate in FP64 and round to or from FP32
 * at the stage boundary); the curl, the tau solves, the influence and sigma
 * corrections, the pressure wall data and the mean-flow update stay FP64.
 * MIXED needs NX2 and NZ2 in {32, 48, 64, 72, 96, 128, 144, 192, 196}. */
typedef enum { CDNS_PRECISION_FP64 = 0, CDNS_PRECISION_MIXED = 1 } cdns_precision;

/* Mesh, mirrors MeshParm (src/core/params.hpp:6-11) + XL/ZL
 * (src/core/mesh.hpp:9-37).  cdns_create holds the whole channel
 * (INDEX_Serial = 1); cdns_pencil_create one rank of a decomposition
 * (INDEX_Serial = 0). */
typedef struct {
    int NX, NY, NZ;
    int NXS, NYS, NZS;
    int NX2, NY2, NZ2;
    double XL, ZL;
} cdns_mesh_desc;

/* Physical and control parameters, mirrors Parm / Control
 * (src/core/params.hpp:13-35) and the derived GRAD_PRE / QXmean values
 * (src/core/params.cpp:296-307, recomputed from THETA). */
typedef struct {
    double Re;
    double G_pre, a_pre0, b_pre0;
    double a_V[3], b_V[3];
    int INDEX_GRAD_PRE;
    double THETA;            /* degrees */
    double DT;
    double V_Microblow0;
} cdns_params;

typedef struct cdns_ctx cdns_ctx;

/* Create a context on CUDA device `device`.  Replaces the construction of
 * Transforms (src/fft/transforms.cpp:59-281), EqSolvePV
 * (src/solver/eqsolve_pv.cpp:132-146) and TimeStepper.  The velocity
 * boundary data starts as velocity_boundary() (src/sim/initial_bc.cpp:95-101). */
int cdns_create(const cdns_mesh_desc *mesh, const cdns_params *params, int precision,
                int device, cdns_ctx **out);
int cdns_destroy(cdns_ctx *ctx);

/* State transfer in the reference layout.  set_velocity also restarts the
 * multistep history (a restart is first order, doc/algorithm.md:104).
 * Replaces FieldIO::read_restart's hand-over (src/io/field_io.cpp:311-427). */
int cdns_set_velocity(cdns_ctx *ctx, const double *velocity);
int cdns_get_velocity(cdns_ctx *ctx, double *velocity);
int cdns_get_pressure(cdns_ctx *ctx, double *pressure);
/* Replace the pressure of the last step (read by cdns_get_pressure and the
 * output reduction; the step itself does not read it). */
int cdns_set_pressure(cdns_ctx *ctx, const double *pressure);
int cdns_set_velocity_bc(cdns_ctx *ctx, const double *bc);
int cdns_set_velocity_device(cdns_ctx *ctx, const double *velocity_dev);
/* Replace the current velocity and keep the multistep history (the previous
 * velocity, nonlinear term and pressure wall data), as the reference's
 * disturbance injection changes velocity_ between two steps of a run
 * (Simulation::apply_disturbance, src/sim/simulation.cpp:96-106, called from
 * Simulation::run :255-256); the next step stays second order.  Whole-channel
 * contexts that already hold a velocity. */
int cdns_update_velocity(cdns_ctx *ctx, const double *velocity);
int cdns_get_velocity_device(cdns_ctx *ctx, double *velocity_dev);

/* One time step of Simulation::run (src/sim/simulation.cpp:174-185,
 * INDEX_Serial = 1): step_coefficients(iteration), EqSolvePV::setup at
 * iteration < 3, enqueue_serial_step and correct_flow.  `iteration` is the
 * 1-based loop counter `it`.  Asynchronous on the context stream;
 * status checks (non-finite values, pivots) are reported by cdns_synchronize. */
int cdns_step(cdns_ctx *ctx, int iteration);

/* `nsteps` steps starting at loop counter `first_iteration`; steps with
 * it >= 3 replay captured CUDA graphs.  Returns after enqueueing. */
int cdns_run(cdns_ctx *ctx, int first_iteration, int nsteps);

/* Wait for the context stream; returns CDNS_ERR_NONFINITE / CDNS_ERR_PIVOT if
 * a step since the last call raised one. */
int cdns_synchronize(cdns_ctx *ctx);

/* Pressure gradient of the last step (dpdx_, dpdz_ of Simulation, used by
 * Statistics::accumulate). */
int cdns_get_dpdx(cdns_ctx *ctx, double out[2]);

/* Nonlinear term alone, TimeStepper::nonlinear_term
 * (src/solver/timestepper.cpp:11-17): N = u x curl u on the product grid and
 * the pressure wall data B [2*NZS+1][2][NXS+1]. */
int cdns_nonlinear(cdns_ctx *ctx, const double *velocity, double *nonlinear, double *pressure_bc);

/* Fine-grid transform of one scalar field, Transforms::channel_xyzfft2
 * (src/fft/transforms.cpp:615-741).  direction 'B': spectral -> physical,
 * 'F': physical -> spectral. */
int cdns_transform_fine(cdns_ctx *ctx, int direction, const double *in, double *out);

/* The fine-grid backward transform of cdns_transform_fine ('B': spectral ->
 * physical, one scalar field) for callers that cannot allocate device
 * memory -- code that runs under a caller-owned memory pool or inside an
 * embedding framework that forbids or intercepts cudaMalloc.  No counterpart
 * in the reference.  `spectral` [2*NZS+1][NYS+1][NXS+1] (complex) and
 * `physical` [NZ2][NY2+1][NX2] are device pointers on the current device;
 * the work is queued on `stream` (a cudaStream_t, NULL for the default
 * stream) and the call returns without waiting.  No context is needed.
 * Intermediate buffers and tables live in one 32 MiB array in device memory
 * that the library holds on every GPU that loads it (product grids up to
 * about 96^3); larger meshes are rejected with CDNS_ERR_ARG.  The array's
 * memory is committed when the library's device code is loaded on a device:
 * at the first call there with lazy module loading (the CUDA default), at
 * library load with eager loading; calls allocate nothing after that.  The
 * first call on each device looks up that array's address, and the first
 * call with a mesh (after a call with another mesh) computes that mesh's
 * tables into the array and raises the kernels' shared-memory limits; make
 * such calls before any stream capture.  Later calls with the same mesh only
 * queue the three transform kernels.  All calls share the array: calls that
 * overlap on the GPU (different streams, threads or devices' streams running
 * at once on one device) race and must be serialised by the caller. */
int cdns_transform_fine_backward_noalloc(const cdns_mesh_desc *mesh, const double *spectral,
                                         double *physical, void *stream);

/* Coarse-grid transform of one scalar field, Transforms::channel_xyzfft
 * (src/fft/transforms.cpp:452-582): direction 'B' spectral [2*NZS+1][NYS+1][NXS+1]
 * -> physical [NZ][NY+1][NX], 'F' the inverse; a full spectrum (NXS = NX/2,
 * NZS = NZ/2) takes the reference's Nyquist halve/mirror convention. */
int cdns_transform_coarse(cdns_ctx *ctx, int direction, const double *in, double *out);

/* The output branch of Simulation::run (src/sim/simulation.cpp:226-235) on
 * the device, for the context's current velocity and pressure:
 * FieldIO::to_physical (src/io/field_io.cpp:199-220), Statistics::reduce
 * (src/sim/statistics.cpp:55-110) and Diagnostics::evaluate
 * (src/sim/diagnostics.cpp:38-80).  Writes, each if not NULL:
 *   plane_sums [NY+1][20]  PlaneMoments::sum per y plane (sums 7..19 zero
 *                          unless higher_moments, as Statistics::reduce);
 *   diagnostics[4]         EKT, TKE, divergence L2, finite (1 or 0);
 *   physical [4][NZ][NY+1][NX]  the snapshot u, v, w, p of to_physical.
 * Only the plane sums (and the snapshot, if asked for) cross to the host;
 * the physical fields are formed and reduced on the GPU.  The reference's
 * Statistics::accumulate(planes, dpdx, dpdz) and Diagnostics::append take
 * these values unchanged. */
int cdns_output_reduce(cdns_ctx *ctx, int higher_moments, double *plane_sums, double *diagnostics,
                       double *physical);

/* Restart and physical-field files in the reference's formats (FieldIO,
 * src/io/field_io.cpp:121-427, single rank), from and into the device state:
 * text = 0 binary v1 (the driver's field_S_ 0.bin / field_P_ 0.bin), 1 text
 * (*.dat).  The restart holds the velocity [..spectral..][3]; the physical
 * file the to_physical snapshot u, v, w, p on the coarse grid.
 * cdns_read_restart takes either form (it probes the magic), checks the
 * header against the mesh and the payload for finite values, and sets the
 * velocity (a first-order restart, as cdns_set_velocity).  Files are written
 * beside the target and renamed over it. */
int cdns_write_restart(cdns_ctx *ctx, const char *path, long long step, double time, int text);
int cdns_read_restart(cdns_ctx *ctx, const char *path, long long *step, double *time);
int cdns_write_physical(cdns_ctx *ctx, const char *path, long long step, double time, int text);

/* Statistics sampling on the device (the `sample` branch of Simulation::run,
 * src/sim/simulation.cpp:227-250).  cdns_statistics_sample queues on the
 * context stream, with no host synchronisation, the reduction of the current
 * state and Statistics::accumulate's running-mean update
 * (src/sim/statistics.cpp:117-139) with the last step's dp/dx and dp/dz.
 * cdns_statistics_read returns the sample count, the (dpdx, dpdz) means and
 * means [20][NY+1]: velocity mean u v w, pressure mean, velocity second
 * moments uu vv ww uv vw wu, pressure second, pressure-velocity pu pv pw,
 * velocity third and fourth moments (u v w each) -- the arrays
 * Statistics::write prints; cdns_statistics_reset starts over. */
int cdns_statistics_sample(cdns_ctx *ctx);
int cdns_statistics_read(cdns_ctx *ctx, long long *count, double *dp_means, double *means);
int cdns_statistics_reset(cdns_ctx *ctx);

/* EqSolvePV::setup(g) followed by the fused solve (solve_modes with fused
 * RHS divergence and sigma correction, src/solver/eqsolve_pv.cpp:311-450)
 * of a given velocity RHS [..][3], pressure wall data [..][2][..] and velocity
 * wall data [..][2][..][3]; writes pressure and velocity and, if `units` is
 * not NULL, u_dpdx_unit then w_dpdz_unit (2*(NYS+1) doubles). */
int cdns_solve(cdns_ctx *ctx, double g, const double *rhs_velocity, const double *pressure_bc,
               const double *velocity_bc, double *pressure, double *velocity, double *units);

/* Launch-shape autotuning (the analogue of FFTW planning and wisdom,
 * src/fft/transforms.cpp:190-278, src/fft/wisdom.cpp:11-32).  An FP64 context
 * picks, at creation, the kx lines per block of its z transforms, the rows per
 * block of its x stage and the form
 * of its Chebyshev synthesis and analysis (FP64 MMA matrix products or one
 * length-NY2 FFT per column), by timing the candidates on its own buffers the
 * first time a mesh is seen on a device in the process (CDNS_TUNE=0 in the
 * environment keeps fixed rules; CDNS_Y_TRANSFORM=matrix|fft fixes the
 * Chebyshev form, CDNS_X_STAGE=rows4|rows2|halfwarp|split|split2 the x-stage
 * form; CDNS_WISDOM=<file> imports that wisdom file once per process
 * and exports to it after each new measurement).  cdns_tune times again; cdns_get_tuning writes
 * {z lines, synthesis FFT form, analysis FFT form, x-stage form} into out[4]
 * (x-stage form: 4 or 2 rows per block, 1 the half-warp form, 3 or 5 the
 * lane-pair split form with 4 or 2 rows);
 * cdns_wisdom_export / _import save and load the choices as JSON (host-only
 * calls); cdns_wisdom_forget empties the process cache. */
int cdns_tune(cdns_ctx *ctx);
int cdns_get_tuning(cdns_ctx *ctx, int *out);
int cdns_wisdom_export(const char *path);
int cdns_wisdom_import(const char *path);
int cdns_wisdom_forget(void);

/* Per-stage device timing for roofline accounting.  Between
 * cdns_profile_begin and cdns_profile_end, steps launch stage by stage on
 * the context stream with CUDA events between stages (no graph replay);
 * cdns_profile_end synchronises and writes the summed milliseconds of each
 * stage into stage_ms[cdns_stage_count()] and the number of steps timed. */
int cdns_profile_begin(cdns_ctx *ctx);
int cdns_profile_end(cdns_ctx *ctx, double *stage_ms, int *nsteps);
int cdns_stage_count(void);
const char *cdns_stage_name(int stage);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or CUDA events against the step. */
int cdns_get_stream(cdns_ctx *ctx, void **stream);

/* Copy an intermediate stage buffer of the last nonlinear evaluation to the
 * host, for stage-by-stage validation: which = 0 Chebyshev-synthesised
 * fields [6][NY2+1][2*NZS+1][NXS+1], 1 z-physical fields
 * [6][NY2+1][NZ2][NXS+1], 2 x-analysed products [3][NY2+1][NZ2][NXS+1]
 * (complex), 3 vorticity wall sums [2][2*NZS+1][NXS+1], 4 solver state
 * summary: per-array count of non-finite values (ad_p, ad_v, influence
 * divergence, sigma0, influence fields, B-problem fields, unit responses)
 * as 7 doubles, 5 normalised influence divergence [2][2][2*NZS+1][NXS+1], 6
 * influence velocities [2][3][..spectral..], 7 influence pressures
 * [2][..spectral..], 8 sigma0 [2][2*NZS+1][NXS+1] (complex), 9 the diagonals
 * wn of the pressure and velocity problems [2][2*NZS+1][NXS+1] (real).
 * `count` is the number of doubles the host buffer holds. */
int cdns_debug_copy(cdns_ctx *ctx, int which, double *out, size_t count);

/* Number of bytes of device memory the context holds. */
int cdns_device_bytes(cdns_ctx *ctx, size_t *bytes);

/* Copy the last error message of the calling thread into buf. */
int cdns_last_error(char *buf, size_t len);

/* Library version string. */
const char *cdns_version(void);

/* Discrete adjoint of the FP64 step (no reference counterpart).
 *
 * cdns_adjoint_run runs iterations 1..nsteps from the context's velocity
 * (a first-order start, as after cdns_set_velocity) with the velocity wall
 * data `control` ([2*NZS+1][2][NXS+1][3] as in cdns_set_velocity_bc; NULL
 * keeps the current data, a non-NULL array becomes the context's data),
 * and evaluates `objective`:
 *   CDNS_OBJECTIVE_WALL_SHEAR  J = (1/nsteps) sum_{n=1..nsteps} tau_w(u^n),
 *     tau_w = (dU/dy(-1) - dU/dy(+1)) / (2 Re) of the streamwise mean
 *     profile U (the (kz, kx) = (0, 0) mode of component 0); `weights` unused.
 *   CDNS_OBJECTIVE_PROJECTION  J = Re sum conj(w) u^nsteps over the stored
 *     coefficients, w = `weights` in the velocity layout: the gradients are
 *     then the vector-Jacobian product of the nsteps-step map with w.
 * If grad_velocity or grad_control is not NULL it also returns the gradient
 * of J with respect to the real and imaginary parts of every stored
 * coefficient of the initial velocity ([..spectral..][3], as cdns_set_velocity)
 * and of the velocity wall data ([..][2][..][3]), by the hand-written
 * transpose of every stage of the step, run backwards over states restored
 * from in-memory checkpoints taken every `checkpoint_interval` steps of the
 * forward sweep (recomputing each interval once).  On return the context
 * holds the state after `nsteps` steps, as after cdns_run(ctx, 1, nsteps).
 * Requires CDNS_PRECISION_FP64, INDEX_GRAD_PRE = 1 and dealiased meshes
 * (NX2 > 2 NXS, NZ2 > 2 NZS, NY2 > NYS). */
#define CDNS_OBJECTIVE_WALL_SHEAR 0
#define CDNS_OBJECTIVE_PROJECTION 1
int cdns_adjoint_run(cdns_ctx *ctx, int nsteps, int checkpoint_interval, int objective,
                     const double *weights, const double *control, double *objective_value,
                     double *grad_velocity, double *grad_control);

/* Transposes of single stages, for tests of the adjoint: the solve of
 * cdns_solve (inputs are the adjoints of its pressure and velocity outputs,
 * outputs the adjoints of its rhs, pressure and velocity wall data, in the
 * same layouts) and the nonlinear term of cdns_nonlinear about `velocity`
 * (adjoints of N and of the pressure wall data in, adjoint of the velocity
 * out).  Under the real inner product Re sum conj(a) b of the stored arrays. */
int cdns_solve_adjoint(cdns_ctx *ctx, double g, const double *pressure_adj, const double *velocity_adj,
                       double *rhs_adj, double *pressure_bc_adj, double *velocity_bc_adj);
int cdns_nonlinear_adjoint(cdns_ctx *ctx, const double *velocity, const double *nonlinear_adj,
                           const double *pressure_bc_adj, double *velocity_adj);

/* Ensemble batch: n independent channels (meshes and params may differ, one
 * precision mode) on one device.  No reference counterpart (the reference
 * runs one channel per process); each member is a full context whose state
 * is set and read with the single-channel calls on cdns_batch_member.
 * cdns_batch_run advances every member from `first_iteration`: steps 1-2 run
 * member by member, steady steps replay one CUDA graph holding every
 * member's step as a parallel branch.  All members must be at the same
 * iteration (set their velocities before the first run). */
typedef struct cdns_batch cdns_batch;
int cdns_batch_create(int n, const cdns_mesh_desc *meshes, const cdns_params *params, int precision,
                      int device, cdns_batch **out);
int cdns_batch_destroy(cdns_batch *batch);
int cdns_batch_size(cdns_batch *batch, int *n);
int cdns_batch_member(cdns_batch *batch, int i, cdns_ctx **ctx);
int cdns_batch_run(cdns_batch *batch, int first_iteration, int nsteps);
/* Waits for every member and reports the first member error (with its index). */
int cdns_batch_synchronize(cdns_batch *batch);
/* The batch's CUDA stream (a cudaStream_t): steady steps are launched on it. */
int cdns_batch_stream(cdns_batch *batch, void **stream);

/* Pencil decomposition of one channel over `ranks` ranks (one GPU each):
 * replaces the reference's distributed path (INDEX_Serial = 0) -- Mesh's
 * block tables (src/core/mesh.cpp:20-85) and the transposes of Transforms
 * (src/fft/transforms.cpp:126-170, 304-404) called from Simulation::run's
 * multi-rank branch (src/sim/simulation.cpp:191-218).
 *
 * Rank r holds the spectral state of the kx block [kx0, kx0 + nkx) (all kz
 * and Chebyshev modes; cdns_set_velocity / cdns_get_velocity /
 * cdns_get_pressure / cdns_set_velocity_bc take the reference layout of that
 * block, [2*NZS+1][..][nkx](+[3])) and, inside a step, the fine-grid y slab
 * [j0, j0 + nj) of the NY2 + 1 points.  Blocks follow the reference's rule:
 * n / ranks each, one more on each of the last n % ranks ranks; ranks must
 * not exceed NXS + 1, NY + 1 or NY2 + 1.  Rank 0 holds the zero mode.
 *
 * cdns_pencil_layout writes table[4 * r ..] = {kx0, nkx, j0, nj} for every
 * rank (host only).  A step of iteration `it` is
 *   cdns_pencil_stage(ctx, it, 0)   curl, Chebyshev synthesis, pack exchange 0
 *   all-to-all of exchange 0         send buffer -> peers' recv buffers
 *   cdns_pencil_stage(ctx, it, 1)   unpack, z synthesis, x stage, z analysis, pack exchange 1
 *   all-to-all of exchange 1
 *   cdns_pencil_stage(ctx, it, 2)   unpack, Chebyshev analysis, column solve
 * on every rank; stages run on the context stream (cdns_get_stream) and the
 * exchange must be ordered on it.  cdns_pencil_buffer gives each exchange's
 * send (recv = 0) or receive (recv = 1) buffer on the device and its length
 * in doubles; the per-peer lengths, in rank order, are cdns_pencil_counts
 * (host only; send[q] on this rank equals recv[rank] on rank q).  Whole-channel
 * calls (cdns_step, transforms, output, files, adjoint) refuse a pencil
 * rank context with CDNS_ERR_STATE.  FP64 only. */
int cdns_pencil_layout(const cdns_mesh_desc *mesh, int ranks, int *table);
int cdns_pencil_counts(const cdns_mesh_desc *mesh, int ranks, int rank, int exchange, long long *send,
                       long long *recv);
int cdns_pencil_create(const cdns_mesh_desc *mesh, const cdns_params *params, int ranks, int rank, int device,
                       cdns_ctx **out);
int cdns_pencil_buffer(cdns_ctx *ctx, int exchange, int recv, void **ptr, long long *doubles);
int cdns_pencil_stage(cdns_ctx *ctx, int iteration, int stage);

/* Fused exchange: instead of pack -> all-to-all -> unpack, stage 1's z
 * synthesis reads its slab's rows of y-physical columns straight from every
 * rank's column buffer and its z analysis writes the nonlinear term back
 * there (plain loads and stores; across GPUs, peer access over NVLink).
 * cdns_pencil_columns gives this rank's column buffer (device pointer and
 * length in doubles); cdns_pencil_set_peers(ctx, columns) takes every rank's,
 * in rank order, as device pointers valid in this process (CUDA IPC or peer
 * mappings across processes; entry `rank` must be this context's own), and
 * NULL returns to the exchange buffers.  With peers set, a step is stage 0 on
 * every rank, then stage 1 once all ranks finished stage 0, then stage 2 once
 * all finished stage 1 (the caller's barrier; no kernel waits on another
 * rank).  Needs NX2 and NZ2 with a register split (32, 48, 64, 72, 96, 128,
 * 144, 192, 196). */
int cdns_pencil_columns(cdns_ctx *ctx, void **ptr, long long *doubles);
int cdns_pencil_set_peers(cdns_ctx *ctx, void *const *columns);
/* Across processes: cdns_pencil_ipc_handle writes the CUDA IPC handle of this
 * rank's column buffer (CDNS_IPC_HANDLE_BYTES bytes, to be sent to the other
 * ranks); cdns_pencil_open_peer maps a peer's handle into this process and
 * returns the device pointer for cdns_pencil_set_peers (unmapped when the
 * context is destroyed). */
#define CDNS_IPC_HANDLE_BYTES 64
int cdns_pencil_ipc_handle(cdns_ctx *ctx, void *handle);
int cdns_pencil_open_peer(cdns_ctx *ctx, const void *handle, void **ptr);
/* Unmap every peer buffer this context opened and return it to the exchange
 * buffers (after waiting for its stream).  Across processes, every rank calls
 * it and then meets the others at a barrier before any rank destroys its
 * context, so that no rank frees a buffer another rank still maps (the
 * teardown order the CUDA IPC API asks for; MpiContext has none to mirror). */
int cdns_pencil_close_peers(cdns_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif /* CDNS_H */
