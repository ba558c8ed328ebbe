/*
 * clipb.h -- C ABI of the B200-native CLIP lattice update (libclipb.so).
 *
 * Drop-in boundary for the per-timestep path of mshadkhah/CLIP.  The reference exposes
 * that path as the C++ class pair Solver <- NSAllen (include/solver/Solver.cuh:37-151,
 * include/equation/NsAllen.cuh:38-126), constructed from InputData/Domain/Geometry/
 * Boundary/DataArray (src/main.cu:53-61) and driven by main's time loop
 * (src/main.cu:74-89).  Each entry point below names the reference call it replaces.
 *
 * Conventions
 *  - Every function returns 0 on success or a negative CLIPB_E* code; clipb_last_error()
 *    gives the message of the last failure on the calling thread.  No C++ exception
 *    crosses this boundary (the reference throws std::runtime_error on config errors and
 *    calls exit(1) on CUDA failures: Logger.cuh:61-67, DataArray.cuh:30-42).
 *  - The library owns all device memory of a solver; one solver is used by one host
 *    thread at a time.  Work is issued on the solver's stream (clipb_set_stream), not on
 *    the legacy default stream; functions that return host data synchronise that stream.
 *  - Host field buffers use the reference's layout unless stated otherwise: the ghosted
 *    extent (2D: (N_x+2) x (N_y+2); 3D: N_x x N_y x N_z, ghosts inside N), x slowest,
 *    component fastest (Domain.cuh:63-68).
 */
#ifndef CLIPB_H
#define CLIPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct clipb_solver clipb_solver;

/* Storage/arithmetic precision of the populations. */
enum {
    CLIPB_FP64 = 0, /* f, g stored and collided in FP64 (parity path)                         */
    CLIPB_FP32 = 1, /* f, g stored and collided in FP32                                       */
    CLIPB_FP16 = 2  /* f, g stored in FP16 as scaled deviations, collided in FP32             */
};

/* Error codes. */
enum {
    CLIPB_OK = 0,
    CLIPB_E_CONFIG = -1,    /* config.txt could not be read or is not supported            */
    CLIPB_E_CUDA = -2,      /* a CUDA call failed                                          */
    CLIPB_E_ARG = -3,       /* bad argument (null pointer, unknown name, size mismatch)    */
    CLIPB_E_STATE = -4,     /* call out of order (e.g. solve before init)                  */
    CLIPB_E_NOMEM = -5,     /* device allocation failed                                    */
    CLIPB_E_DIVERGED = -6   /* a monitor found NaN (Reporter.cu:141-142)                   */
};

/* Field identifiers for clipb_get_field / clipb_set_field. */
enum {
    CLIPB_FIELD_C = 0,      /* order parameter c (phi)            1 component             */
    CLIPB_FIELD_P = 1,      /* pressure p = sum f_post            1 component             */
    CLIPB_FIELD_RHO = 2,    /* density rho = rhoL + c (rhoH-rhoL)  1 component             */
    CLIPB_FIELD_VEL = 3,    /* velocity u                         DIM components          */
    CLIPB_FIELD_F = 4,      /* post-collision f (reference dev_f) Q components            */
    CLIPB_FIELD_G = 5,      /* post-collision g (reference dev_g) Q components            */
    CLIPB_FIELD_F_POST = 6, /* streamed + bounced f (dev_f_post)  Q components            */
    CLIPB_FIELD_G_POST = 7  /* streamed + bounced g (dev_g_post)  Q components            */
};

typedef struct clipb_info {
    int dim;              /* 2 or 3                                                        */
    int q;                /* 9 (D2Q9) or 19 (D3Q19)                                        */
    int precision;        /* CLIPB_FP64 / FP32 / FP16                                      */
    int extent[3];        /* ghosted extent in the reference's convention                  */
    int interior[3];      /* interior node counts                                          */
    long long steps;      /* time steps taken since init                                   */
    size_t device_bytes;  /* device memory held by the solver                              */
    double pop_scale;     /* FP16 only: power-of-two scale of the stored f deviations       */
} clipb_info;

/* Parse a CLIP config.txt and allocate a solver.
 * Replaces InputData(config) + Domain + Geometry + Boundary + DataArray(createVectors) +
 * NSAllen(...) (src/main.cu:53-61; InputData.cu:43-115, Domain.cu:22-82,
 * Geometry.cu:50-58, Boundary.cu:25-32, DataArray.cu:79-121, NsAllen.cu:47-56). */
int clipb_create(const char* config_path, int precision, clipb_solver** out);

/* Free every resource of the solver.  Replaces ~DataArray (DataArray.cu:48-75). */
void clipb_destroy(clipb_solver* s);

/* Message of the last failed call on this thread ("" if none). */
const char* clipb_last_error(void);

/* Parse a config.txt without touching the GPU: dimension, reference extent (3 ints),
 * boundary code per side (6 ints: 0 wall, 1 slip wall, 2 free convect, 3 periodic, 4 neumann,
 * 5 velocity, -1 absent) and the 16
 * derived parameters of clipb_get_params.  Any pointer may be NULL.  Replaces the
 * parsing half of InputData/Boundary/Geometry (InputData.cu:57-115, Boundary.cu:146-319,
 * Geometry.cu:72-203). */
int clipb_config_summary(const char* config_path, int* dim, int* extent3, int* sides6, double* params16);

/* Issue all further work of the solver on this CUDA stream (a cudaStream_t; NULL selects
 * the solver's own non-blocking stream).  No reference counterpart: the reference uses
 * the legacy default stream throughout. */
int clipb_set_stream(clipb_solver* s, void* cuda_stream);

int clipb_get_info(const clipb_solver* s, clipb_info* out);

/* Step counts of the config: finalStep, outputInterval, reportInterval, checkpointInterval
 * (4 values; 0 where the config has none).  Mirrors the interval fields of
 * InputData::params (InputData.cu:57-67), which TimeInfo, VTSwriter, Reporter and
 * CheckPointer read. */
int clipb_get_intervals(const clipb_solver* s, long long* out4);

/* checkpointCopy of the config (0 where it has none): how many earlier checkpoint folders
 * CheckPointer keeps beside the newest (CheckPointer.cu:53-64, 108-138); 0 disables
 * checkpoints in the reference's loop. */
int clipb_get_checkpoint_copies(const clipb_solver* s, long long* copies);

/* Host-to-device bytes of the last initial-field upload (clipb_init or
 * clipb_device_initializer; 0 after clipb_init_device).  Large fields send, per z plane,
 * only the rows from the first to the last that is not uniform with the plane's edge rows,
 * plus a small per-plane table; the uniform rows are written on the device.  The
 * reference copies the whole field (NsAllen::deviceInitializer, NsAllen.cu:897-908). */
int clipb_get_upload_bytes(const clipb_solver* s, long long* bytes);

/* Derived parameters in the order RhoL RhoH sigma muH muL tauH tauL kConstant betaConstant
 * mobility interfaceWidth referenceLength gx gy gz caseType (16 doubles).
 * Mirrors InputData::params after read_config (InputData.cu:57-115). */
int clipb_get_params(const clipb_solver* s, double* out16);

/* Host initial phase field from the geometry's signed distance (c over the ghosted
 * extent, reference layout).  Replaces NSAllen::initialCondition (NsAllen.cu:768-824).
 * c_out may be NULL (the field is then only kept inside the solver). */
int clipb_initial_condition(clipb_solver* s, double* c_out);

/* Upload c (NULL: the field of clipb_initial_condition) and build the initial state:
 * chemical potential, gradient, normal and equilibrium populations, then the first
 * collision.  Replaces DataArray::updateDevice + NSAllen::deviceInitializer
 * (DataArray.cu:124-128, NsAllen.cu:897-908). */
int clipb_device_initializer(clipb_solver* s, const double* c_host);

/* clipb_initial_condition + clipb_device_initializer. */
int clipb_init(clipb_solver* s);

/* The same initial state with the initial field evaluated on the GPU (FP64, one thread per
 * node) instead of on the host: no host loop and no upload, for large grids.  The field
 * differs from the host evaluation only where CUDA's tanh and the C library's tanh round
 * differently (a few units in the last place); clipb_init stays the path that equals the
 * reference bit for bit.  Replaces NSAllen::initialCondition + DataArray::updateDevice +
 * NSAllen::deviceInitializer (NsAllen.cu:768-824, 897-908; DataArray.cu:124-128). */
int clipb_init_device(clipb_solver* s);

/* Advance nsteps time steps (asynchronous on the solver's stream).
 * Replaces nsteps calls of NSAllen::solve (NsAllen.cu:881-892). */
int clipb_solve(clipb_solver* s, int nsteps);

/* Copy a field to host memory in the reference layout (ghosted extent, x slowest,
 * components fastest).  Interior values are the solver's state; ghost cells hold the
 * values the reference would hold after the same step where the path defines them.
 * Replaces DataArray::updateHost / copyFromDevice (DataArray.cu:131-138). */
int clipb_get_field(clipb_solver* s, int field, double* host_out, size_t count);

/* Copy c, p, rho and u to host in one call (any pointer may be NULL): the body of
 * VTSwriter::writeToFile's per-step updateHost (VTSwriter.cu:72-79). */
int clipb_get_fields(clipb_solver* s, double* c, double* p, double* rho, double* u);

/* Interior fields only, x fastest, components as separate planes (SoA), copied into a
 * caller-provided DEVICE buffer on the solver's stream (no host round trip). */
int clipb_get_field_device(clipb_solver* s, int field, double* dev_out, size_t count);

/* Mass sum(c) and kinetic energy sum(0.5 rho |u|^2) over the interior, FP64 on the GPU.
 * Replaces Reporter::sum (Reporter.cu:95-114; its per-call cudaMalloc/free and its
 * double counting of the last block's tail are not reproduced).  Returns
 * CLIPB_E_DIVERGED if either is NaN (Reporter.cu:141-142). */
int clipb_monitors(clipb_solver* s, double* mass, double* kinetic);

/* nsteps steps (>= 1) and the monitors of the state they leave, as clipb_solve followed by
 * clipb_monitors, with the reduction folded into the last step: on the 3D direct-load
 * launch variants that step sums the mass and kinetic energy of each row segment of 32
 * nodes as it stores c and u, and two short passes add those partials in a fixed order, so
 * the stored state is not read again.  The result does not depend on the launch variant or
 * the planes per CTA; it differs from clipb_monitors' only by the order of the FP64
 * additions (within 1e-13 relative).  The staged variants, cases with free-convect or
 * Neumann sides and 2D cases run clipb_solve and clipb_monitors.  CLIPB_E_DIVERGED on NaN, as clipb_monitors (Reporter.cu:124-144). */
int clipb_solve_monitored(clipb_solver* s, int nsteps, double* mass, double* kinetic);

/* Time nsteps of clipb_solve with CUDA events on the solver's stream; *ms receives the
 * elapsed device time.  No reference counterpart (the reference has no timers). */
int clipb_time_steps(clipb_solver* s, int nsteps, float* ms);

/* Launch shape of the fused step: `variant` selects a tile shape / register policy
 * (0 .. nvariants-1), `seg` the planes (3D) or rows (2D) each thread block marches over
 * (0 = default: 2D takes the longest of 16, 8, 4, 2 rows that leaves eight blocks per SM).  Results do not depend on the launch shape.  No reference counterpart
 * (the reference launches fixed 8x8(x4) blocks, DataArray.cu:27-44). */
int clipb_set_launch(clipb_solver* s, int variant, int seg);
int clipb_get_launch(const clipb_solver* s, int* variant, int* seg, int* nvariants);

/* Time every launch shape on the solver's freshly initialised state (trial_steps each),
 * keep the fastest, and rebuild the initial state.  Any output pointer may be NULL;
 * *ms_per_step receives the winner's time per step. */
int clipb_autotune(clipb_solver* s, int trial_steps, int* variant, int* seg, float* ms_per_step);

/* Bounded waits of the staged 3D step (launch variants 5 and 6): each wait for a bulk copy
 * gives up after `cycles` SM clock cycles (0 = the default, 2^31, about a second), sets the
 * solver's device error flag and lets the block drain its copies and return; the flag makes
 * clipb_monitors, clipb_get_field and clipb_time_steps fail with CLIPB_E_CUDA.
 * inject_bytes > 0 is a test hook of that path: the first bulk load of every block then
 * expects that many bytes more than its copies bring, so its wait runs out (no fault, no
 * hang: the block completes the missing bytes itself before it drains).  No reference
 * counterpart (the reference has no bulk copies and never checks a launch). */
int clipb_set_wait_limit(clipb_solver* s, long long cycles, unsigned inject_bytes);

/* clipb_solve replays a captured CUDA graph of 16 steps when it is asked for more than 16
 * steps (default on); enable = 0 issues one launch per step instead.  enable = 1 on an
 * initialised solver (and clipb_autotune) captures the graph at once, so that the first
 * long clipb_solve does not spend host time on it. */
int clipb_set_graphs(clipb_solver* s, int enable);

/* Mass sum(c) and kinetic energy sum(rho |u|^2 / 2), rho = rho_l + c * drho, of n nodes
 * held in caller-owned DEVICE arrays (dev_c: n values; dev_u: dim planes of n values, e.g.
 * the output of clipb_get_field_device), written to the caller-owned device array
 * dev_out2 (2 doubles) on `stream` (NULL: the legacy default stream).  The call then waits
 * for the two sums and returns CLIPB_E_DIVERGED when either is NaN, like clipb_monitors.
 * The blocks sum a flat grid-stride range of the dense arrays, not clipb_monitors' rows of
 * the device layout, so the two agree to rounding, not bit for bit.
 *
 * No counterpart in the reference.  For callers that cannot allocate device memory when
 * they need the monitors (an arena or pool owning the device, allocation-free real-time
 * loops, hosts that pass only their own buffers): this entry point calls no cudaMalloc,
 * cudaFree or other allocating routine.  Its per-block partial sums live in a fixed array
 * in the library's device image (2 x 1024 doubles, held by every GPU that loads the
 * library until the process exits); nblocks (0 = 4 per SM of the device, at most 1024)
 * must not exceed 1024, larger values are rejected with CLIPB_E_ARG.  The first call in
 * each device context looks up that array's device address and the SM count (with the
 * device current), so make the first call before any stream capture; a context recreated
 * after cudaDeviceReset is detected by its id and looked up again.  Calls share the array;
 * calls whose kernels overlap on the GPU race on it. */
int clipb_field_sums_noalloc(const double* dev_c, const double* dev_u, int dim, long long n, double rho_l,
                             double drho, double* dev_out2, int nblocks, void* stream);

/* ---------------------------------------------------------------- VTS output
 * File <folder>/<base_name>_t<step>.vts (step = the solver's step count; the folder is
 * created): a VTK structured grid over the interior nodes with the point arrays Velocity
 * (DIM components), C, P and Rho, as VTSwriter::writeVTSBinaryFile writes it
 * (VTSwriter.cu:84-205).  Values equal those of clipb_get_fields at the same nodes.
 *   CLIPB_VTS_ASCII     the reference's text file (Float64 values printed as %g, 6
 *                       significant digits, like its default-formatted std::ofstream)
 *   CLIPB_VTS_BINARY64  the same arrays as raw little-endian Float64 in an appended block
 *                       (VTK XML 1.0, UInt64 block headers)
 *   CLIPB_VTS_BINARY32  the same as Float32: half the copy and the file
 * The reference copies every field to the host on every step (DataArray::updateHost in
 * VTSwriter::writeToFile) to write one step in outputInterval.  Here a kernel packs the
 * interior fields on the solver's stream; the device-to-host copy (own stream, pinned
 * buffers) and the file write (a writer thread) overlap the following steps. */
enum { CLIPB_VTS_ASCII = 0, CLIPB_VTS_BINARY64 = 1, CLIPB_VTS_BINARY32 = 2 };

/* Queue the write of the current state and return once its pack kernel is enqueued.  At
 * most two writes are in flight per solver; a third call waits for the oldest. */
int clipb_write_vts_async(clipb_solver* s, const char* folder, const char* base_name, int format);

/* Wait for every queued write of the solver; returns the first failure among them
 * (CLIPB_E_ARG with the file name when a file could not be written). */
int clipb_vts_wait(clipb_solver* s);

/* clipb_write_vts_async + clipb_vts_wait. */
int clipb_write_vts(clipb_solver* s, const char* folder, const char* base_name, int format);

/* ---------------------------------------------------------------- z slabs (several GPUs)
 * No counterpart in the reference, which runs one case on one GPU (multi-GPU is on its
 * roadmap, README.md:249).  A 3D case is split into slabs of whole z planes, one per GPU;
 * each slab is an ordinary solver (clipb_solve, clipb_monitors, clipb_get_field, ...) whose
 * step updates only its own planes.  On each face that borders another slab it keeps the
 * neighbour's boundary plane and the plane beyond it; before every step (and after
 * clipb_init) the caller moves one packet per face: clipb_slab_pack on the neighbour,
 * any device-to-device transport (NCCL send/recv, a peer copy), clipb_slab_unpack here.
 * With that exchange the owned planes evolve exactly as in the whole case (bit for bit).
 * Slabs take wall, slip-wall and periodic sides; the step must be taken one step at a time
 * (clipb_solve(s, 1), or its two parts) with the exchange in between. */

/* A solver for global planes z_begin .. z_end (1-based, at least 2) of the 3D case in
 * config_path.  exchange_faces: bit 0 = the z- face borders another slab, bit 1 = the z+
 * face does.  Faces inside the case must be exchange faces; on a periodic z axis either
 * both faces are (several slabs) or the slab holds the whole axis.  clipb_init,
 * clipb_autotune and clipb_load set the slab's state including its copies of the
 * neighbours' planes: exchange after each of them before the next step.  Monitors and VTS
 * files cover the slab's own planes (VTS at their global z). */
int clipb_slab_create(const char* config_path, int precision, int z_begin, int z_end, int exchange_faces,
                      clipb_solver** out);

/* The slab's global planes, its own planes in local numbering (zlo .. zhi, as clipb_get_field
 * numbers them) and the bytes of one face packet.  Any pointer may be NULL. */
int clipb_slab_info(const clipb_solver* s, int* z_begin, int* z_end, int* zlo, int* zhi, long long* packet_bytes);

/* Write into dev_packet (device memory of packet_bytes) the planes that the neighbour on
 * side `toward` (0: z-, 1: z+) needs before the next step: f, g and c of this slab's
 * boundary plane on that side, g and c of the plane inside it.  Asynchronous on `stream`
 * (a cudaStream_t; NULL: the solver's stream), which must be ordered after the step. */
int clipb_slab_pack(clipb_solver* s, int toward, void* dev_packet, void* stream);

/* Write a packet received from the neighbour on side `face` (0: z-, 1: z+) into this
 * slab's planes on that face.  Asynchronous on `stream` (NULL: the solver's stream); the
 * next step must be ordered after it. */
int clipb_slab_unpack(clipb_solver* s, int face, const void* dev_packet, void* stream);

/* One step of a slab in two parts, so that its packets travel while the rest of the step
 * runs.  Part 1 updates the owned planes that clipb_slab_pack reads (the two next to each
 * face; every plane of a slab of at most 4); part 2 updates the others and completes the
 * step.  Between the parts only clipb_slab_pack and clipb_slab_unpack may be called (on
 * another stream, ordered after part 1): they read and write planes that part 2 does not
 * touch.  Parts 1 and 2 equal clipb_solve(s, 1) bit for bit.  Both parts run on the
 * solver's stream. */
int clipb_slab_step_part(clipb_solver* s, int part);

/* Write a checkpoint folder: the files of the reference's CheckPointer::save
 * (src/io/CheckPointer.cu:53-80: dev_f/dev_g/dev_f_post/dev_g_post.bin as FP64 arrays in
 * the reference layout, timeInfo.bin, domainSize.bin, info.txt), readable by the
 * reference's CheckPointer::load, plus clipb_state.bin with libclipb's exact state. */
int clipb_save(clipb_solver* s, const char* dir);

/* Resume from a checkpoint folder (CheckPointer::load, CheckPointer.cu:85-101): bit-exact
 * from clipb_state.bin (same precision and grid); from the reference's files alone, the
 * last step is replayed from dev_f/dev_g with c rebuilt exactly and the previous velocity
 * approximated by sum e_q f_post (the reference saves neither c nor u). */
int clipb_load(clipb_solver* s, const char* dir);

/* ---------------------------------------------------------------- derivatives (2D, FP64)
 * Objective J = |X(c_N) - target|^2 with X = sum(x c) / sum(c) over the interior nodes
 * (x: node coordinates in the reference's ghosted index convention), after nsteps steps of
 * the FP64 forward from the initial c field c0 (reference layout over the ghosted extent;
 * NULL: the config's initial condition).  Parameters, in this order: the body-force
 * acceleration g_y, the surface tension sigma (with kappa = 1.5 sigma W, beta = 8 sigma/W
 * and the initial pressure jump; InputData.cu:108-109, NsAllen.cu:768-824) and the
 * mobility M (w_c = 1/(1/2 + 3M), NsAllen.cu:549).  Walls and periodic sides.
 * No counterpart in the reference, which has no derivatives. */

/* Set g_y, sigma and M (and the parameters derived from them) of an FP64 or any solver. */
int clipb_set_params(clipb_solver* s, double gy, double sigma, double mobility);

/* J after a forward run (init from c0, then nsteps steps); leaves the solver at step nsteps. */
int clipb_objective(clipb_solver* s, const double* c0, int nsteps, const double* target2, double* J);

/* Tangent-linear model: J and its directional derivative dJ for the perturbation dc0
 * (reference layout, NULL: 0) of c0 and dparams3 (NULL: 0) of (g_y, sigma, M). */
int clipb_tangent(clipb_solver* s, const double* c0, int nsteps, const double* target2, const double* dc0,
                  const double* dparams3, double* J, double* dJ);

/* Adjoint: J, its gradient with respect to c0 (reference layout over the ghosted extent,
 * may be NULL) and to (g_y, sigma, M) (may be NULL).  The forward states are recomputed
 * from checkpoints taken every `checkpoint_every` steps; checkpoint_every >= nsteps keeps
 * every state of the run in one tape instead (no recomputation).  0: one tape when its
 * nsteps + 1 states take at most half of the free device memory (with the workspace the
 * solver already holds), else checkpoints every 100 steps.  Device memory: one tape of
 * K + 1 states (two with more than one segment), a checkpoint per segment, about 60
 * adjoint planes; it stays with the solver for later calls.  Leaves the solver at step
 * nsteps, as clipb_objective does.  No reference counterpart (the reference has no
 * derivatives). */
int clipb_adjoint(clipb_solver* s, const double* c0, int nsteps, const double* target2, int checkpoint_every,
                  double* J, double* grad_c0, double* grad_params3);

/* ---------------------------------------------------------------- batched 2D cases
 * Many independent 2D cases advanced together: one persistent launch per time step over
 * a packed table of every case's step arguments and a list of work items (case, tile,
 * row segment), replayed from a CUDA graph.  No counterpart in the reference, which runs
 * one case per process (src/main.cu:39-92); each case has exactly the semantics of a
 * single solver created from the same config (clipb_create), with the same results bit
 * for bit.  Cases must be 2D with wall and periodic sides. */
typedef struct clipb_batch clipb_batch;

enum {
    CLIPB_CONFIG_PATH = 0, /* configs[i] is the path of a config.txt                        */
    CLIPB_CONFIG_TEXT = 1  /* configs[i] is the text of a config.txt                        */
};

/* Parse ncases configs (paths or texts) and allocate every case. */
int clipb_batch_create(const char* const* configs, int ncases, int kind, int precision, clipb_batch** out);
void clipb_batch_destroy(clipb_batch* b);
int clipb_batch_size(const clipb_batch* b);

/* Borrowed handle of case `index` (owned by the batch; do not destroy): every clipb_get_*
 * query and clipb_monitors work on it.  Its work runs on the batch's stream. */
int clipb_batch_case(clipb_batch* b, int index, clipb_solver** out);

/* Initial state of every case (clipb_init per case). */
int clipb_batch_init(clipb_batch* b);

/* Advance every case by nsteps: one batched launch per step (graph replay of 16 steps
 * for longer runs). */
int clipb_batch_solve(clipb_batch* b, int nsteps);

/* The same steps as plain per-case launches, one case after another (the baseline the
 * batched launch is measured against; identical results). */
int clipb_batch_solve_sequential(clipb_batch* b, int nsteps);

/* Launch shape of the batched step: 2D tile variant (as clipb_set_launch), rows per work
 * item, persistent thread blocks per SM (0: as many as fit).  Results do not depend on it. */
int clipb_batch_set_launch(clipb_batch* b, int variant, int rows_per_item, int blocks_per_sm);
int clipb_batch_get_launch(const clipb_batch* b, int* variant, int* rows_per_item, int* blocks_per_sm, int* nitems);

/* Time every launch shape on the freshly initialised batch, keep the fastest and rebuild
 * the initial state (outputs may be NULL; *ms_per_step: the winner's time per step). */
int clipb_batch_autotune(clipb_batch* b, int trial_steps, int* variant, int* rows_per_item, int* blocks_per_sm,
                         float* ms_per_step);
int clipb_batch_set_graphs(clipb_batch* b, int enable);

/* Device time of nsteps (sequential != 0: clipb_batch_solve_sequential). */
int clipb_batch_time_steps(clipb_batch* b, int nsteps, int sequential, float* ms);

/* Per-case mass and kinetic energy (arrays of clipb_batch_size entries; either may be NULL). */
int clipb_batch_monitors(clipb_batch* b, double* mass, double* kinetic);

/* Config text of case `index` of the seeded batch workload (host only, no GPU): drop and
 * bubble alternating; N_x in {32..256} and N_y in {64..512} in steps of 32, We ~ U[1,20],
 * Re ~ U[50,500], rhoRatio log-uniform on [10,1000], muRatio = rhoRatio/10,
 * R = 0.2 min(N_x, N_y), referenceLength = 2R, mobility 0.02, W = 4, g = (0,-1e-6,0),
 * periodic x, walls y.  Drawn from std::mt19937_64(seed): per case, in this order,
 * N_x = 32 (1 + r % 8), N_y = 64 + 32 (r % 15), then three uniforms (r >> 11) / 2^53 for We,
 * Re and log rhoRatio.  Writes at most len bytes (NUL-terminated) and returns the full text
 * length. */
int clipb_seeded_case_config(unsigned long long seed, int index, char* buf, size_t len);

#ifdef __cplusplus
}
#endif

#endif /* CLIPB_H */
