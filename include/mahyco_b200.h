/*
 * mahyco_b200.h -- C ABI of the B200 MaHyCo hydro-cycle library
 * (libmahyco_b200.so).  Plain pointers and sizes only.
 *
 * Every entry point returns an int status: 0 = MHC_OK, < 0 = API error,
 * > 0 = numerical status flags of the case (a bitwise OR of MHC_ST_*).
 * The reference reports the same numerical conditions by exit(1) or
 * stopComputeLoop; here they are returned so that a failing case can be
 * retired without stopping the process.
 *
 * Reference interfaces replaced (file:line inside cea-hpc/MaHyCo):
 *   module entry points      src/Mahyco.axl:244-261, src/MahycoModule.h:164-349
 *   time loop order          src/Mahyco.config:15-36
 *   IEquationOfState         src/eos/IEquationOfState.h:38-65
 *   IRemap                   src/Remap/IRemap.h:44-63
 *   EnvSummation time history src/time_history/EnvSummationService.cc:77-169
 */
#ifndef MAHYCO_B200_H
#define MAHYCO_B200_H

#include "mahyco_case.h"

#ifdef __cplusplus
extern "C" {
#endif

/* API errors */
#define MHC_OK 0
#define MHC_ERR_ARG (-1)          /* bad argument / unknown name */
#define MHC_ERR_CUDA (-2)         /* CUDA runtime error (message: mhc_last_error) */
#define MHC_ERR_UNSUPPORTED (-3)  /* option outside the implemented hot path */
#define MHC_ERR_ORDER (-4)        /* entry point called out of time-loop order */
#define MHC_ERR_NOMEM (-5)        /* device allocation failed / HBM budget */

/* numerical status flags (returned as positive values) */
#define MHC_ST_NEG_VOLUME 1       /* MahycoModule.cc:1164-1191 (exit(1) there) */
#define MHC_ST_DT_UNDERFLOW 2     /* MahycoModule.cc:1816-1833 (exit(1) there) */
#define MHC_ST_NAN 4              /* RemapADIFinal.cc:274-284 (exit(1) there) */
#define MHC_ST_STOP 8             /* final time reached: stopComputeLoop (MahycoModule.cc:1851-1857) */
#define MHC_ST_OOM_ADMISSION 16   /* serving: the case does not fit the HBM budget */
#define MHC_ST_TIMEOUT 32         /* serving: the request outlived its deadline */
#define MHC_ST_DAMAGE 64          /* Endommagement: a cell met a damage threshold (damaged cells are not modelled) */

typedef struct mhc_case mhc_case;

/* last error message of the calling thread (static storage) */
const char* mhc_last_error(void);

/* library version string */
const char* mhc_version(void);

/* Case lifecycle.  Allocates the device state of one case on the current
 * CUDA device, on a private stream.  Replaces the Arcane module instance. */
int mhc_case_create(const mhc_case_params* params, mhc_case** out);
int mhc_case_destroy(mhc_case* h);

/* the CUDA stream (cudaStream_t) every kernel of the case is launched on,
 * so that callers can record events or order their own work after it */
void* mhc_case_stream(mhc_case* h);

/* Checkpoint / restart of the device-resident state (protection-reprise,
 * MahycoModule.cc:273-308): every device field, the time-loop scalars and
 * the host-side loop state of a case, copied to a host buffer of
 * mhc_case_checkpoint_bytes(h) bytes between iterations; a restore into a
 * case created with identical parameters continues bit-identically.
 * MHC_ERR_ORDER in the middle of an iteration, MHC_ERR_ARG for a buffer
 * of another case or layout. */
long long mhc_case_checkpoint_bytes(mhc_case* h);
int mhc_case_checkpoint(mhc_case* h, void* host, long long capacity);
int mhc_case_restore(mhc_case* h, const void* host, long long size);

/* Fills *p with the reference option defaults (src/Mahyco.axl:263-557,
 * Remap/RemapADI.axl:162-210, the EOS .axl files; a PerfectGas environment,
 * SOD case model, one environment, a 1x1x1 3D mesh on the unit cube) for a
 * host that then sets the options of its .arc dataset.  Host only. */
void mhc_case_params_default(mhc_case_params* p);
/* sizeof(mhc_case_params) as this library was built, for bindings that
 * mirror the structure (no device work) */
long long mhc_case_params_size(void);

/* HBM bytes one case with these parameters needs (serving admission). */
long long mhc_case_device_bytes(const mhc_case_params* params);

/* --- init entry points (Mahyco.config:15-21) ----------------------------
 * HydroStartInit + ComputeCellMass + ComputeNodeMass
 * (MahycoModule.cc:21-262, MahycoAnnexe.cc:11-235). */
int mhc_hydro_start_init(mhc_case* h);

/* --- compute-loop entry points (Mahyco.config:23-36) --------------------
 * They must be called in time-loop order.  Consecutive entry points are
 * fused into one kernel launch; a fused stage is launched by its last
 * entry point:
 *   SaveValuesAtN  (no device work: values at n stay in place)
 *   UpdateVelocity, ApplyBoundaryCondition, UpdatePosition      -> node pass
 *   ComputeGeometricValues, UpdateDensity, ComputeArtificialViscosity,
 *   UpdateElasticityAndPlasticity, UpdateEnergyAndPressure       -> cell pass
 *   Remap                                                        -> ADI remap
 *   ComputeDeltaT                                                -> dt reduction */
int mhc_save_values_at_n(mhc_case* h);
int mhc_update_velocity(mhc_case* h);
int mhc_apply_boundary_condition(mhc_case* h);
int mhc_update_position(mhc_case* h);
int mhc_compute_geometric_values(mhc_case* h);
int mhc_update_density(mhc_case* h);
int mhc_compute_artificial_viscosity(mhc_case* h);
int mhc_update_elasticity_and_plasticity(mhc_case* h);
int mhc_update_energy_and_pressure(mhc_case* h);
int mhc_remap(mhc_case* h);
int mhc_compute_delta_t(mhc_case* h);

/* n complete compute-loop iterations, enqueued asynchronously on the case
 * stream (no host synchronisation inside).  Iterations after a stop or an
 * error flag are skipped on the device. */
int mhc_cycle(mhc_case* h, int n);

/* same as mhc_cycle, but the iterations are captured once in a CUDA graph
 * (one 6-iteration period, which brings every sweep order back) and
 * replayed; n = 0 right after HydroStartInit captures the graph without
 * running an iteration */
int mhc_cycle_graph(mhc_case* h, int n);

/* kernel groups of one iteration, for mhc_cycle_timed */
enum mhc_stage {
  MHC_STAGE_LAGRANGE_NODES = 0,  /* velocity, BC, position */
  MHC_STAGE_LAGRANGE_CELLS = 1,  /* geometry, density, pseudo, energy */
  MHC_STAGE_SWEEP_CELLS = 2,     /* one remap direction, cells */
  MHC_STAGE_SWEEP_NODES = 3,     /* one remap direction, dual (nodes) */
  MHC_STAGE_FINALIZE_CELLS = 4,  /* remapVariables + EOS */
  MHC_STAGE_FINALIZE_NODES = 5,  /* node velocity and mass */
  MHC_STAGE_DELTA_T = 6,         /* CFL reduction */
  MHC_NUM_STAGES = 7
};

/* mhc_cycle with CUDA events recorded on the case stream around every
 * kernel group; stage_ms[s] receives the summed device time of stage s,
 * stage_launches[s] (optional) its number of launches.  Synchronises after
 * each group, so use it for measurement, not production. */
int mhc_cycle_timed(mhc_case* h, int n, double* stage_ms, long long* stage_launches);

/* wait for the case stream; returns the numerical status flags */
int mhc_synchronize(mhc_case* h);

/* time-loop scalars after the last completed iteration */
int mhc_get_scalars(mhc_case* h, double* time, double* deltat, long long* iteration, int* status);
/* asynchronous status read-back: mhc_scalars_request enqueues, after the
 * work already on the case stream, a copy of the scalars into one of two
 * pinned host slots and returns the slot (0 or 1, alternating);
 * mhc_scalars_wait blocks until that copy has landed and returns its values
 * (same meaning as mhc_get_scalars).  A time loop can enqueue iteration k+1,
 * then wait for the scalars of iteration k, so the GPU never idles on the
 * read-back. */
int mhc_scalars_request(mhc_case* h);
int mhc_scalars_wait(mhc_case* h, int slot, double* time, double* deltat, long long* iteration, int* status);

/* Named fields (names of src/Mahyco.axl: Density, Pressure, InternalEnergy,
 * SoundSpeed, PseudoViscosity, CellMass, CellVolume, FracVol, MassFraction,
 * CaracteristicLength, EnvMask, Temperature (Lagrangian runs; the cell value
 * of a mixed cell is 0, as the services write environment values only),
 * StrainTensorXX/YY/ZZ/XY/YZ/XZ, PlasticDeformation,
 * PlasticDeformationVelocity, StrainNorm (elasto-plastic runs); nodes:
 * Velocity (x,y,z interleaved),
 * NodeMass, NodeCoord, and VelocityN for sans-lagrange cases: the prescribed
 * velocities at n).  env < 0 selects the global cell value, env >= 0
 * the environment value (0 where the cell is not in the environment).
 * Returns the number of doubles written, or an error. */
long long mhc_get_field(mhc_case* h, const char* name, int env, double* host, long long capacity);

/* Initial fields, before mhc_hydro_start_init: what the reference reads
 * from the dataset's mesh file and <initialisation> block.  NodeCoord (3
 * per node, x y z interleaved, the library's node order): the initial
 * positions of a Lagrangian case, a mesh file's grid (mahyco_b200/msh.py
 * maps the logically structured Gmsh quadrangle grids of the datasets);
 * Materiau, Density, Pressure (one per cell): the initial state of the
 * EXTERNAL case model (the values not given: environment 0 and its
 * initial state).  Returns the number of doubles read, or an error. */
long long mhc_case_set_initial_field(mhc_case* h, const char* name, const double* host, long long n);

/* Upload of a named field, the inverse of mhc_get_field, so that a host can
 * push its own state onto the device (a restart from its own dumps, an
 * initialisation this library lacks, a hand-off from its CPU code).  Same
 * names, env semantics and layout as mhc_get_field: env < 0 writes the
 * global cell value; env >= 0 writes the environment value of the cells
 * that hold env (the global slot for the cells where env is alone, as the
 * reference's environment manager stores them) and ignores the others.
 * EnvMask (bit e = environment e present) is written as given: set it
 * before the environment values.  CellVolume takes env < 0 only;
 * NodeCoord is derived geometry (the corner normals of the last Lagrangian
 * mesh are kept with it) and is read-only.  Only between iterations (after
 * HydroStartInit, MHC_ERR_ORDER otherwise).  Reads n doubles of host;
 * returns the number read, or an error.  Replaces the writes a host makes
 * through Arcane's variables (src/Mahyco.axl:6-241). */
long long mhc_set_field(mhc_case* h, const char* name, int env, const double* host, long long n);

/* --- IEquationOfState (IEquationOfState.h:38-65) ------------------------
 * One call per method of the service interface, on environment env of the
 * case (its .axl options are the mhc_env_params of that environment).
 * mhc_eos_apply: applyEOS(env) on the current density and internal energy
 * of the env cells; mixed cells holding env then get computePressionMoyenne.
 * The temperature (field "Temperature", carried by Lagrangian runs) is set by
 * mhc_eos_init and advanced by the iterations; mhc_eos_apply and
 * mhc_eos_apply_one_cell leave it (its update needs the energy at the start
 * of the iteration, which is not kept between iterations). */
int mhc_eos_apply(mhc_case* h, int env);
/* initEOS(env): internal energy and sound speed of the env cells from their
 * pressure and density (PerfectGasEOSService.cc:12-35,
 * StiffenedGasEOSService.cc:14-33, MieGruneisenEOSService.cc:12-34) */
int mhc_eos_init(mhc_case* h, int env);
/* ReinitEOS(env): the three services restore nothing on a restart (their
 * ReinitEOS bodies are empty); checks its arguments and returns */
int mhc_eos_reinit(mhc_case* h, int env);
/* applyOneCellEOS(env, EnvCell): pressure and sound speed of one cell of
 * env written in place, dp/de returned in *dpde (may be NULL); the cell
 * must hold env.  Synchronous (reads dp/de back). */
int mhc_eos_apply_one_cell(mhc_case* h, int env, long long cell, double* dpde);
/* Endommagement(env): the damage test of the services on every env cell
 * (pressure below tension-damage-thresold, or density / initial density
 * below density-damage-thresold).  The library accepts only the default
 * thresholds, under which no cell of positive density and pressure above
 * the threshold is damaged, and does not model damaged cells: a cell that
 * meets the test sets MHC_ST_DAMAGE on the case (which then stops). */
int mhc_eos_endommagement(mhc_case* h, int env);
/* getAdiabaticCst(env), getdensityDamageThresold(env) */
int mhc_eos_get_adiabatic_cst(mhc_case* h, int env, double* out);
int mhc_eos_get_density_damage_thresold(mhc_case* h, int env, double* out);

/* --- IRemap (IRemap.h:44-63) ---------------------------------------------
 * mhc_remap_apply: the remap stage of the current iteration
 * (appliRemap, which ends with remapVariables), for a caller that has run
 * the Lagrange entry points. */
int mhc_remap_apply(mhc_case* h);
/* appliRemap(dimension, withDualProjection, nb_vars_to_project, nb_env)
 * with the reference's arguments, checked against the case: dimension and
 * nb_env those of the case, withDualProjection 1 (the only form the
 * reference's module uses), nb_vars_to_project 18 nb_env
 * (MahycoAnnexe.cc:65) or 3 nb_env + 5 after a restart (MahycoModule.cc:288).
 * The library projects its own packed set (3 nb_env + 1 cell and 5 node
 * quantities), whatever the count. */
int mhc_remap_appli_remap(mhc_case* h, int dimension, int with_dual_projection, int nb_vars_to_project, int nb_env);
/* the two halves of appliRemap: the direction sweeps
 * (RemapADIService.cc:23-56), then the Euler reset and remapVariables
 * (RemapADIService.cc:58-87, RemapADIFinal.cc:21-346); same arguments */
int mhc_remap_sweeps(mhc_case* h);
int mhc_remap_variables(mhc_case* h, int dimension, int with_dual_projection, int nb_vars_to_project, int nb_env);
/* resizeRemapVariables(nb_vars_to_project, nb_env): the remap arrays are
 * sized when the case is created; checks the counts as appliRemap does */
int mhc_remap_resize_remap_variables(mhc_case* h, int nb_vars_to_project, int nb_env);
/* synchronizeUremap(): ghost-layer exchange between sub-domains; one case
 * lives on one device here, so there is nothing to exchange */
int mhc_remap_synchronize_uremap(mhc_case* h);
/* option getters: the value (>= 0), or an error (< 0) */
int mhc_remap_get_ordre_projection(mhc_case* h);
int mhc_remap_has_projection_pente_borne(mhc_case* h);
int mhc_remap_has_projection_simple_pente(mhc_case* h);
int mhc_remap_has_conservation_energie_totale(mhc_case* h);
/* isEuler(): "Full", "X", "Y" or "Z" copied into out (capacity bytes) */
int mhc_remap_is_euler(mhc_case* h, char* out, int capacity);

/* --- EnvSummation (EnvSummationService.cc:77-169) -----------------------
 * out[0] = time, then per environment: CellMass (plain average), Pressure
 * (plain average), Density (volume weighted), InternalEnergy (mass
 * weighted), present flag: 1 + 5*nb_env doubles. */
int mhc_time_history(mhc_case* h, double* out);

/* --- batches: many independent cases, one launch per phase ---------------
 * No counterpart in the reference (which runs one case per process).  All
 * cases of a batch live on the device at once; mhc_batch_cycle advances
 * every active case by n iterations with one persistent launch per kernel
 * phase over a work list that covers all their blocks, whatever their mesh
 * sizes.  A case stops advancing once it reaches its iteration limit, its
 * final time or an error flag; its neighbours are unaffected.  Results are
 * bit-identical to the same case run alone. */
typedef struct mhc_batch mhc_batch;
int mhc_batch_create(mhc_batch** out);
/* the same on a stream the caller owns (a cudaStream_t, e.g. created with a
 * priority); it must outlive the batch */
int mhc_batch_create_on_stream(void* stream, mhc_batch** out);
int mhc_batch_destroy(mhc_batch* b);
void* mhc_batch_stream(mhc_batch* b);
/* add a case (device state allocated, not yet initialised); iteration_limit
 * <= 0 means unlimited; *index identifies the case in this batch */
int mhc_batch_add(mhc_batch* b, const mhc_case_params* params, long long iteration_limit, int* index);
/* HydroStartInit of every case added since the last call */
int mhc_batch_init(mhc_batch* b);
/* retire a case and release its device memory */
int mhc_batch_remove(mhc_batch* b, int index);
int mhc_batch_cycle(mhc_batch* b, int n);
/* same, replaying a CUDA graph of 6 iterations (one sweep-rotation period) */
int mhc_batch_cycle_graph(mhc_batch* b, int n);
int mhc_batch_cycle_timed(mhc_batch* b, int n, double* stage_ms, long long* stage_launches);
int mhc_batch_synchronize(mhc_batch* b);
/* launch grid of the phases: 0 (default) = one block per work item,
 * k > 0 = k x the blocks the device can hold at once, striding the list */
int mhc_batch_set_grid_scale(mhc_batch* b, int scale);
/* per-phase override of the grid scale (stage = enum mhc_stage, scale -1 =
 * back to the batch-wide value); the autotuner sets these */
int mhc_batch_set_stage_grid_scale(mhc_batch* b, int stage, int scale);
/* layout of the y / z remap sweeps of classical-limiter cases, for cells
 * and for nodes: 0 = by mesh size (default), 1 = one warp per line,
 * 2 = shared-memory tile, 3 = one thread per line chunk.  Results are the
 * same bit for bit whatever the layout; the autotuner picks the fastest.
 * The _case_ variants set them, and the per-phase grid scale, for one case
 * run alone. */
int mhc_batch_set_sweep_layout(mhc_batch* b, int cell_layout, int node_layout);
int mhc_case_set_sweep_layout(mhc_case* h, int cell_layout, int node_layout);
int mhc_case_set_stage_grid_scale(mhc_case* h, int stage, int scale);
/* number of kernels the batch (or a single case) has put on the GPU so far;
 * a CUDA graph replay counts every kernel node it runs */
long long mhc_batch_launches(mhc_batch* b);
long long mhc_case_launches(mhc_case* h);
int mhc_batch_get_scalars(mhc_batch* b, int index, double* time, double* deltat, long long* iteration, int* status);
long long mhc_batch_get_field(mhc_batch* b, int index, const char* name, int env, double* host, long long capacity);
/* stop advancing a case but keep its state resident (fields stay readable
 * until mhc_batch_remove) */
int mhc_batch_detach(mhc_batch* b, int index);
/* checkpoint / restart of one case of a batch (see mhc_case_checkpoint) */
long long mhc_batch_checkpoint_bytes(mhc_batch* b, int index);
int mhc_batch_checkpoint(mhc_batch* b, int index, void* host, long long capacity);
int mhc_batch_restore(mhc_batch* b, int index, const void* host, long long size);
/* iteration done, status flags and time of every case index (removed: -1),
 * read with one gather kernel and one copy; returns the number of indices */
int mhc_batch_poll(mhc_batch* b, int capacity, long long* iteration, int* status, double* time);
/* the same without waiting: mhc_batch_poll_request enqueues the gather and
 * the copy after the work already on the batch stream and returns a request
 * id (0 or 1, alternating; two may be outstanding); mhc_batch_poll_wait
 * waits for that copy and fills the arrays as mhc_batch_poll does (cases
 * added after the request: iteration 0, status 0).  A host can enqueue the
 * next cycles, then read the previous status while they run. */
int mhc_batch_poll_request(mhc_batch* b);
int mhc_batch_poll_wait(mhc_batch* b, int request, int capacity, long long* iteration, int* status, double* time);

/* --- serving: continuous batching under an HBM budget --------------------
 * No counterpart in the reference (one case per process there).  Requests
 * (a case and an iteration count) are queued by submit; every step admits
 * queued requests whose device footprint (mhc_case_device_bytes) fits the
 * budget, in arrival order with bounded backfilling, advances the resident
 * cases with one launch per phase and size class (the slowest class
 * `cycles` iterations, smaller classes as many as take about as long,
 * at most 64 x cycles), and retires
 * the cases that reached their iteration count, stopped or failed.  Results
 * stay resident, and charged to the budget, until released.  Per-request
 * status: the MHC_ST_* flags, including MHC_ST_OOM_ADMISSION (larger than
 * the whole budget) and MHC_ST_TIMEOUT (deadline exceeded). */
typedef struct mhc_server mhc_server;
enum { MHC_REQ_QUEUED = 0, MHC_REQ_RUNNING = 1, MHC_REQ_DONE = 2, MHC_REQ_FAILED = 3 };
/* budget <= 0: 90% of the device memory free at creation */
int mhc_server_create(long long hbm_budget_bytes, mhc_server** out);
int mhc_server_destroy(mhc_server* s);
/* requests are served by size class (cells < 3e4, < 1e6, larger), each a
 * batch on its own stream; the larger the class, the higher its stream's
 * priority, so a large request is not slowed by small ones sharing the
 * GPU; stream of class cls (0..2) */
void* mhc_server_stream(mhc_server* s, int cls);
/* kernels the server has put on the GPU so far */
long long mhc_server_launches(mhc_server* s);
/* timeout_s <= 0: no deadline */
int mhc_server_submit(mhc_server* s, const mhc_case_params* p, long long iterations, double timeout_s, long long* ticket);
/* admits what fits, enqueues `cycles` iterations (per class, see above)
 * and a status read of every class, then waits for the previous step's
 * status read -- the GPU runs this step while the host retires the
 * requests that finished in the previous one; returns the number of
 * requests that completed (done or failed), whose tickets
 * mhc_server_take_completed hands out */
int mhc_server_step(mhc_server* s, int cycles);
/* tickets of the requests completed since the last call (at most capacity;
 * returns how many were written) */
int mhc_server_take_completed(mhc_server* s, long long* tickets, int capacity);
int mhc_server_poll(mhc_server* s, long long ticket, int* state, int* status, long long* iteration, double* time);
/* host clock (seconds since server creation) of submission, admission, completion (-1: not yet) */
int mhc_server_times(mhc_server* s, long long ticket, double* submit, double* admit, double* done);
long long mhc_server_fetch(mhc_server* s, long long ticket, const char* name, int env, double* host, long long capacity);
/* frees a finished request's device state (MHC_ERR_ORDER while queued or running) */
int mhc_server_release(mhc_server* s, long long ticket);
int mhc_server_stats(mhc_server* s, long long* queued, long long* running, long long* bytes_in_use, long long* budget);

/* --- allocation-free CFL time step --------------------------------------
 * No counterpart in the reference: an extra entry point for callers that
 * cannot allocate device memory -- host codes that own all of their device
 * memory through their own pool (as mesh frameworks do), or that run where
 * allocation is not allowed -- and therefore cannot create a case.  It
 * computes the deltat of computeDeltaT (MahycoModule.cc:1739-1833) from the
 * caller's device buffers: cell char_length and sound_speed [ncell], node
 * velocity components vx, vy, vz [nnode] (cartesian numbering, x fastest),
 * and writes the new deltat to deltat_out[0] (device memory): cfl * min
 * l/(c + vmax), bounded by 1.05*old_deltat and deltat_max; -2 when below
 * deltat_min.  vmax, the largest speed of a cell's nodes, enters only when
 * euler_full is non-zero, as computeDeltaT adds it only when the remap's
 * is-euler-scheme is "Full" (MahycoModule.cc:1771; "Full" is the option's
 * default, Lagrangian runs included); with euler_full = 0 the velocity
 * buffers are not read and may be NULL.  deltat-constant runs need no
 * reduction and are not served here.  Work is enqueued on `stream`
 * (a cudaStream_t, or NULL).
 *
 * Bad cells: when any cell gives NaN or a negative l/(c + vmax), the result
 * is -1 and no deltat is produced.  This differs from mhc_compute_delta_t,
 * which sets MHC_ST_NAN on the case, leaves that cell out of the minimum and
 * still produces a deltat from the others.
 *
 * It calls no allocator: the per-block minima live in a fixed array inside
 * the library (MHC_NOALLOC_SCRATCH_BYTES on every GPU that loads it, until
 * the process exits), so meshes above MHC_NOALLOC_MAX_CELLS cells are
 * rejected with MHC_ERR_ARG.  The first call on a device looks the array's
 * address up (cudaGetSymbolAddress); make that first call outside any
 * stream capture.  The address is kept for the life of the process and
 * does not survive a cudaDeviceReset of that device.  All calls on a device
 * share the array: calls that overlap on the GPU race and must be
 * serialised by the caller.
 * Errors: mhc_noalloc_last_error(). */
#define MHC_NOALLOC_MAX_CELLS (1 << 22)
#define MHC_NOALLOC_SCRATCH_BYTES (MHC_NOALLOC_MAX_CELLS / 256 * 8)
int mhc_cfl_delta_t_noalloc(int dim, int nx, int ny, int nz, const double* char_length,
                            const double* sound_speed, const double* vx, const double* vy,
                            const double* vz, int euler_full, double cfl, double old_deltat,
                            double deltat_max, double deltat_min, double* deltat_out, void* stream);
const char* mhc_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
