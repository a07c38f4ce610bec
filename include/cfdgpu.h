/* cfdgpu.h -- C ABI of the B200 (sm_100a) split finite-volume solver for the
 * 2D Euler equations and the Allaire five-equation two-material model.
 *
 * This is the drop-in boundary for cfd-art's time-stepping loop.  A caller
 * that today drives the reference through its plugin interface
 *   problem_base          euler_equations/euler_simulation_code/headers/problem_base.hpp:18-40
 *   splitting_scheme_base euler_equations/euler_simulation_code/headers/splitting_scheme.hpp:22-27
 *   simulation            euler_equations/euler_simulation_code/headers/simulation.hpp:36-67
 * binds the functions below instead (see each declaration for the reference
 * member it replaces).  Plain C types only; every function returns CFD_OK or a
 * negative error code, and cfd_last_error() gives the message.
 *
 * Grids exchanged with the host use the reference's own layout unless stated
 * otherwise: CFD_LAYOUT_GHOSTED_AOS is gridtype (headers/typedefs.hpp:19-21)
 * flattened row-major, (ny + 2g) rows x (nx + 2g) cells x nvar doubles, with
 * g = 2 ghost layers for MUSCL-Hancock and 1 for Godunov
 * (sourcecode/euler_io.cpp:448-461), nvar = 4 (rho, rho u, rho v, E) for
 * Euler and 6 (z rho1, (1-z) rho2, rho u, rho v, E, z) for Allaire.
 */
#ifndef CFDGPU_H
#define CFDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CFD_OK 0
#define CFD_ERR_INVALID (-1)     /* bad argument or configuration */
#define CFD_ERR_CUDA (-2)        /* CUDA runtime error (no device, launch failure, ...) */
#define CFD_ERR_NOMEM (-3)       /* device or host allocation failed */
#define CFD_ERR_STATE (-4)       /* call out of order (e.g. step before upload) */
#define CFD_ERR_UNSUPPORTED (-5) /* option not available in this build */
#define CFD_ERR_BUDGET (-6)      /* request exceeds the device-memory budget */

enum { CFD_MODEL_EULER = 0, CFD_MODEL_ALLAIRE = 1 };
/* CFD_PREC_FP64: plain FP64, bit-identical to the reference.
 * CFD_PREC_MIXED: FP32 arithmetic with an FP32 compensation word per stored
 *   component (batch members and the server).
 * CFD_PREC_FP64_FAST: FP64 arithmetic with contracted multiply-adds and
 *   refined hardware reciprocals / square roots; matches the reference to a
 *   relative L1 density error far below 1e-12, not bit for bit (batch members
 *   and the server). */
enum { CFD_PREC_FP64 = 0, CFD_PREC_MIXED = 1, CFD_PREC_FP64_FAST = 2 };
enum { CFD_BC_TRANSMISSIVE = 0, CFD_BC_REFLECTIVE = 1 };
enum { CFD_LIM_MINMOD = 0, CFD_LIM_VANLEER = 1, CFD_LIM_MC = 2, CFD_LIM_UNLIMITED = 3 };
enum { CFD_FLUX_MUSCL = 0, CFD_FLUX_GODUNOV = 1 };
enum { CFD_SPLIT_NAIVE = 0, CFD_SPLIT_STRANG = 1 };
enum { CFD_WS_DAVIS = 0, CFD_WS_PVRS = 1 };
/* CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE: cfd_download only, ghost cells as the
 * reference's grid holds them at the same point (see cfd_set_reference_ghosts). */
enum { CFD_LAYOUT_GHOSTED_AOS = 0, CFD_LAYOUT_SOA = 1, CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE = 2 };
enum { CFD_BC_LEFT = 0, CFD_BC_RIGHT = 1, CFD_BC_BOTTOM = 2, CFD_BC_TOP = 3 };

/* Event counters (cfd_status.counters); the reference prints or asserts. */
enum {
    CFD_CNT_UNPHYSICAL_INPUT = 0,  /* stencil state failing flux_solver_MUSCLhancock.hpp:131-134 */
    CFD_CNT_SLOPE_ZEROED = 1,      /* flux_solver_MUSCLhancock.hpp:184-189 */
    CFD_CNT_FIRST_ORDER = 2,       /* flux_solver_MUSCLhancock.hpp:216-223 */
    CFD_CNT_FIXUP = 3,             /* sourcecode/euler_rowsweep.cpp:49-81 */
    CFD_CNT_UNPHYSICAL_OUTPUT = 4  /* sourcecode/allaire_diffuse_rowsweep.cpp:49 */
};

/* Problem description.  Replaces the fields of sim_info
 * (headers/sim_info.hpp:16-36) plus the EOS parameters (SGparams /
 * binarySGparams, headers/stiffened_gas_eos.hpp:20-63) and the solver choices
 * read from settingsfile.txt (headers/settings_file.hpp:19-72). */
typedef struct cfd_config {
    int model;            /* CFD_MODEL_* */
    int precision;        /* CFD_PREC_* */
    int nx, ny;           /* interior cells along x (columns) and y (rows), >= 2 */
    double x0, y0, dx, dy;
    double gamma1, pinf1; /* material 1 (Euler: the gas) */
    double gamma2, pinf2; /* material 2 (Allaire) */
    int bc[4];            /* CFD_BC_* per CFD_BC_LEFT..TOP */
    double cfl;           /* CFL number (clamped to 0.2 for the first 5 steps) */
    double T;             /* end time; the time loop stops at t >= T */
    int limiter;          /* CFD_LIM_*; the reference uses minmod */
    int flux_solver;      /* CFD_FLUX_* */
    int splitting;        /* CFD_SPLIT_* */
    int wavespeed;        /* CFD_WS_* (Allaire HLLC wave-speed estimate) */
    double z_min;         /* Allaire: clip z to [z_min, 1 - z_min]; 0 = the reference's [0, 1] */
    int fix_dy_halfstep;  /* 1: y-sweep half step uses dy (reference: dx, euler_colsweep.cpp:43) */
    void* stream;         /* cudaStream_t to run on; NULL: the solver creates its own */
} cfd_config;

/* Snapshot of the device-resident time-loop state. */
typedef struct cfd_status {
    int n;                /* steps taken */
    int done;             /* t >= T */
    double t;             /* simulated time */
    double dt_next;       /* dt compute_dt would return now (device rule) */
    double maxu, maxv;    /* max(|u|+c), max(|v|+c) of the current state */
    double mass1, mass2;  /* sum of rho*dx*dy (Allaire: of each partial density) */
    unsigned long long counters[8];
} cfd_status;

typedef struct cfd_solver cfd_solver;

/* Library identification (build string).  No counterpart in the reference. */
const char* cfd_version(void);

/* Message of the last failing call on this thread; returns its length.
 * Replaces the reference's assert aborts and printed messages (e.g.
 * sourcecode/euler_io.cpp:232). */
int cfd_last_error(char* buf, size_t len);

/* Number of stored components per cell for a model (4 or 6): the vectype
 * size of gridtype (sourcecode/euler_io.cpp:494, A/sourcecode/
 * allaire_diffuse_io.cpp:462). */
int cfd_nvar(int model);

/* Bytes of device memory cfd_create would allocate for cfg.  No counterpart
 * in the reference (host memory only). */
int cfd_device_bytes(const cfd_config* cfg, size_t* bytes);

/* Allocates a solver and its device state.  Replaces problem->set_ICs'
 * storage allocation (sourcecode/euler_io.cpp:494) and the construction of
 * the flux/Riemann solver objects (:466-491). */
int cfd_create(const cfd_config* cfg, cfd_solver** out);
int cfd_destroy(cfd_solver* s);

/* Copies an initial condition to the device and computes the wave speeds of
 * it.  `host` is read in `layout`; ghost cells are ignored (they are rebuilt
 * by every sweep, as pre_sweep does).  n and t set the step count and time.
 * Replaces handing set_ICs' grid to the time loop (headers/simulation.hpp:39-40). */
int cfd_upload(cfd_solver* s, const double* host, int layout, int n, double t);

/* Same from device memory (SoA planes of nx*ny doubles each, nvar planes).
 * No counterpart in the reference. */
int cfd_upload_device(cfd_solver* s, const double* dev_soa, int n, double t);

/* Builds the initial condition on the device, straight into the solver's
 * state: a seeded recipe (CFD_RECIPE_*, declared in cfdgpu_host.h) or a named
 * reference test case (set_ICs, sourcecode/euler_io.cpp:436-731 and
 * A/sourcecode/allaire_diffuse_io.cpp:402-640).  The result is bit-identical
 * to cfd_recipe_ic / cfd_case_ic followed by cfd_upload, without a host grid
 * or a host-to-device copy of the state.  For the four Allaire cases with
 * per-cell formulas (shocked_SF6, TSTM, RMI_SF6, tin_air_implosion), which
 * call sin / cos / atan2, the device's values of those functions decide the
 * rare sample point that lies within an ulp of an interface.  No
 * counterpart in the reference, which builds every grid on the host. */
int cfd_upload_recipe(cfd_solver* s, int recipe, uint64_t seed, int nbubbles, int n, double t);
int cfd_upload_case(cfd_solver* s, const char* test_case, uint64_t seed, int n, double t);

/* Copies the current state to the host in `layout`.  In the ghosted layout
 * the ghost strips hold the boundary fill of the current state.  Replaces
 * reading the grid that problem->output gets (headers/simulation.hpp:50, :65). */
int cfd_download(cfd_solver* s, double* host, int layout);
/* Schlieren field of the current state computed on the device: |grad rho|
 * of every interior cell by central differences, as the reference's writer
 * forms it (E/sourcecode/euler_io.cpp:1142-1185, A/sourcecode/
 * allaire_diffuse_io.cpp:1109-1150), the same values as the host writer's,
 * nx*ny doubles from the bottom row up.  `ghosts` picks the outside
 * neighbours of edge cells like cfd_download's layouts:
 * CFD_LAYOUT_GHOSTED_AOS (boundary fill of the current state) or
 * CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE (the reference's ghost values).  Only
 * nx*ny doubles cross to the host instead of the ghosted grid;
 * cfd_write_schlieren_field normalises and writes them. */
int cfd_schlieren(cfd_solver* s, int ghosts, double* host);

/* Checkpoint / resume.  cfd_checkpoint_save writes the current state, the
 * device time-loop state (n, t, the dt chosen for the next step, wave speeds,
 * masses), the event counters and the reference ghost values when kept, to a
 * binary file (little-endian header + FP64 SoA planes); cfd_checkpoint_load
 * reads it into a solver of the same model, grid and spacing, after which
 * the solve continues bit for bit as if it had not stopped.  Synchronous.
 * No counterpart in the reference, which runs each problem start to end. */
int cfd_checkpoint_save(cfd_solver* s, const char* path);
int cfd_checkpoint_load(cfd_solver* s, const char* path);
/* Reads a checkpoint's header (plain FP64 or batch member): its
 * configuration, step count and time.  Host only. */
int cfd_checkpoint_info(const char* path, cfd_config* cfg, int* n, double* t);

/* Keeps the ghost values the reference's grid holds between boundary fills,
 * for output writers that read ghost cells (the schlieren stencil at the
 * domain edge, the Allaire lineouts): after an upload, the uploaded grid's
 * own ghosts (the initial condition evaluated there, for the device
 * builders; the boundary fill for the SoA layouts); after a step, the fill
 * pre_sweep (sourcecode/euler_ppsweep.cpp:7-118) made before the last sweep
 * that read the buffer now current (naive splitting: the step's x sweep;
 * Strang: its y sweep); corners keep their initial values, as
 * set_boundary_conditions never writes them.  Each step then launches one
 * small extra kernel.  cfd_download with CFD_LAYOUT_GHOSTED_AOS_AS_REFERENCE
 * returns these ghosts.  Enable before the upload to keep its ghost values. */
int cfd_set_reference_ghosts(cfd_solver* s, int enable);

/* problem_base::compute_dt (sourcecode/euler_timestep.cpp:7-44): dt for step
 * n at time t from the current state.  Synchronises the solver's stream. */
int cfd_compute_dt(cfd_solver* s, int n, double t, double* dt_out);

/* splitting_scheme_base::advance_timestep (headers/splitting_scheme.hpp:26):
 * one split step with the given dt (asynchronous on the solver's stream). */
int cfd_step(cfd_solver* s, double dt);

/* The time loop of headers/simulation.hpp:48-61 run on the device: up to
 * max_steps steps with dt chosen on the device after each step, stopping at
 * t >= T.  Asynchronous; steps past the end are no-ops. */
int cfd_advance(cfd_solver* s, int max_steps);

/* Waits for the solver's stream and returns the time-loop state: the n and t
 * that headers/simulation.hpp:44-61 keeps on the host, with the masses
 * compute_dt records (sourcecode/euler_timestep.cpp:31-32) and the counters. */
int cfd_get_status(cfd_solver* s, cfd_status* st);

/* Kernel timing for profiling (no counterpart: the reference times the whole
 * run, sourcecode/main.cpp:39-43): while enabled, every sweep launch is
 * bracketed by CUDA events on the solver's stream (steps launch one by one
 * instead of from the captured graph).  cfd_kernel_times returns the summed
 * durations (ms) and launch counts per sweep direction (0: x, 1: y) since
 * the last reset; it synchronises the stream. */
int cfd_set_kernel_timing(cfd_solver* s, int enable);
int cfd_kernel_times(cfd_solver* s, double ms[2], int launches[2]);
int cfd_reset_kernel_times(cfd_solver* s);

/* Resets the event counters (the reference prints each event instead,
 * e.g. sourcecode/euler_rowsweep.cpp:51). */
int cfd_reset_counters(cfd_solver* s);

/* Waits for all work queued on the solver's stream.  No counterpart in the
 * reference. */
int cfd_synchronize(cfd_solver* s);

/* Device-side layout of the current state for zero-copy callers: SoA planes
 * `plane` elements apart, rows `pitch` elements apart, FP64.  No counterpart
 * in the reference. */
int cfd_state_device(cfd_solver* s, const void** dev_ptr, int64_t* plane, int* pitch);

/* compute_dt without any device allocation, for callers that may not call
 * cudaMalloc: a host application or framework that owns every device
 * allocation through its own pool or a fixed budget, or a latency-critical
 * loop that cannot take the device-wide synchronisation cudaMalloc and
 * cudaFree imply.  No counterpart in the reference: it is the
 * reference's compute_dt (sourcecode/euler_timestep.cpp:7-44) computed on a
 * state the caller already holds on the device.
 *   dev_state: SoA FP64 planes (nvar planes `plane` elements apart, rows
 *              `pitch` elements apart), e.g. from cfd_state_device.
 *   dev_out:   5 device doubles the caller owns, receiving dt (for step n at
 *              time t, cfg's CFL and T), max(|u|+c), max(|v|+c) and the two
 *              mass sums times dx*dy.
 * The per-row reduction scratch is a fixed array inside the library,
 * cfd_noalloc_max_rows() rows (8192) deep and 256 KiB in size, which every GPU
 * that loads the library holds until exit; grids with more rows are rejected
 * with CFD_ERR_INVALID.  Every call shares that array and it keeps the last
 * call's contents, so calls that overlap on the GPU (concurrent streams or
 * threads) race: serialise them.  The configuration is checked as
 * cfd_create checks it (CFD_ERR_INVALID on a bad CFL, spacing or gamma).  The
 * first call on each device looks up the array's device address with that
 * device current and loads the kernels of both models; make that first call
 * before any stream capture.  Asynchronous on `stream` (NULL: the legacy
 * default stream); allocates nothing and frees nothing. */
int cfd_compute_dt_noalloc(const cfd_config* cfg, const double* dev_state, int64_t plane,
                           int pitch, int n, double t, double* dev_out, void* stream);
int cfd_noalloc_max_rows(void);

/* ---- batched solves (mixed and fast FP64 forms) ----------------------------
 * Many independent solves of uneven sizes advanced together: each tick runs
 * one persistent x-sweep launch and one y-sweep launch per model and form
 * over the tiles of every active member, every member choosing its own dt
 * and stopping on its own (at t >= T or after max_steps).  A member's form is
 * its cfg.precision: CFD_PREC_FP64_FAST gives the fast FP64 form (FP64
 * arithmetic with contracted multiply-adds and refined hardware reciprocals
 * and square roots, relative L1 density error far below 1e-12 against the
 * reference), any other value the mixed form: FP32 reconstruction and
 * Riemann solves, state stored as FP32 plus an FP32 compensation word, FP64
 * for stiffened-gas pressure recovery, the CFL reduction and time.  Both
 * take 8 bytes per stored component.  No counterpart in the reference, which runs one
 * problem per process (euler_equations/euler_simulation_code/sourcecode/main.cpp:17-49).
 * Members are admitted against a device-memory budget (bytes; 0 = 80 % of the
 * free memory at creation); cfd_batch_add returns CFD_ERR_BUDGET when a
 * member does not fit. */
typedef struct cfd_batch cfd_batch;
int cfd_batch_create(void* stream, size_t device_budget_bytes, cfd_batch** out);
int cfd_batch_destroy(cfd_batch* b);
/* Device bytes one member of cfg would take. */
int cfd_batch_member_bytes(const cfd_config* cfg, size_t* bytes);
/* Adds a solve from a ghosted AoS initial grid (cfg.splitting must be
 * naive); max_steps <= 0 runs to T.  Synchronous; returns the member id. */
int cfd_batch_add(cfd_batch* b, const cfd_config* cfg, const double* host_ic, int max_steps,
                  int* id_out);
/* Same with the initial condition built on the device from a seeded recipe
 * (see cfd_upload_recipe). */
int cfd_batch_add_recipe(cfd_batch* b, const cfd_config* cfg, int recipe, uint64_t seed,
                         int nbubbles, int max_steps, int* id_out);
int cfd_batch_remove(cfd_batch* b, int id);
/* Saves a member (configuration, FP32 value and compensation planes, time
 * state, step limit) to a checkpoint file; cfd_batch_restore adds it back,
 * to this or another batch, continuing bit for bit (max_steps < 0: the
 * saved step limit).  Lets a server evict a solve and resume it later. */
int cfd_batch_save(cfd_batch* b, int id, const char* path);
int cfd_batch_restore(cfd_batch* b, const char* path, int max_steps, int* id_out);
int cfd_batch_size(cfd_batch* b, int* count, size_t* used_bytes, size_t* budget_bytes);
/* Advances every member by `ticks` steps (members that are done idle). */
int cfd_batch_step(cfd_batch* b, int ticks);
/* Same, one launch at a time with CUDA events: summed x- and y-sweep ms. */
int cfd_batch_step_timed(cfd_batch* b, int ticks, double* ms_x, double* ms_y, int* launches);
/* Autotuner: tries each tile shape per model and sweep direction on real
 * steps (results do not depend on the tiling) and keeps the fastest. */
int cfd_batch_autotune(cfd_batch* b, int steps_per_trial, double* best_tick_ms);
int cfd_batch_set_shapes(cfd_batch* b, int model, int shape_x, int shape_y);
int cfd_batch_get_shapes(cfd_batch* b, int model, int* shape_x, int* shape_y);
/* Strip length of the marching y sweep (y shape 3) of a model: rows in
 * [16, 64], or 0 (default) to choose it for every tile list so that the
 * strips fill the resident warps.  cfd_batch_get_march_rows reports the
 * length the current tile list uses (0 when the model's y sweep does not
 * march or the model has no active member).  Results do not depend on it. */
int cfd_batch_set_march_rows(cfd_batch* b, int model, int rows);
int cfd_batch_get_march_rows(cfd_batch* b, int model, int* rows);
/* Rows of the x sweep's warp-segment tiles (28 columns each) in the current
 * tile list of a model and form (precision CFD_PREC_MIXED or
 * CFD_PREC_FP64_FAST): in [12, 32], chosen for every tile list so that the
 * tiles fill the resident warps; 0 when that model and form have no active
 * member.  Results do not depend on it. */
int cfd_batch_get_segment_rows(cfd_batch* b, int model, int precision, int* rows);
int cfd_batch_status(cfd_batch* b, int id, cfd_status* st);
/* ids, steps taken, done flags and times of all members (cap entries). */
int cfd_batch_poll(cfd_batch* b, int cap, int* ids, int* steps, int* done, double* t, int* count);
/* The same status read in two phases, for callers that queue the next steps
 * before reading: _issue queues the gather behind the work queued so far and
 * returns; _collect waits for that gather and returns what it saw, like
 * cfd_batch_poll (members added after the issue are not in it; count = 0
 * when nothing was issued).  One read may be outstanding at a time. */
int cfd_batch_poll_issue(cfd_batch* b);
int cfd_batch_poll_collect(cfd_batch* b, int cap, int* ids, int* steps, int* done, double* t,
                           int* count);
int cfd_batch_download(cfd_batch* b, int id, double* host, int layout);

/* ---- continuous-batching server --------------------------------------------
 * Clients submit solves from any thread; a worker thread owns the GPU and,
 * between rounds of `ticks_per_round` steps, admits queued requests in
 * arrival order as device memory frees up (requests that do not fit yet keep
 * their place without blocking smaller ones), advances every admitted solve
 * together (mixed: one cfd_batch; FP64: one cfd_solver each on the worker's
 * stream) and hands finished grids back.  No counterpart in the reference. */
enum { CFD_REQ_QUEUED = 0, CFD_REQ_RUNNING = 1, CFD_REQ_DONE = 2, CFD_REQ_FAILED = 3 };

typedef struct cfd_server_options {
    int precision;          /* CFD_PREC_MIXED, CFD_PREC_FP64_FAST (batched) or CFD_PREC_FP64 */
    size_t budget_bytes;    /* device memory for resident solves; 0: budget_fraction */
    double budget_fraction; /* of the free device memory at creation (0: 0.8) */
    int ticks_per_round;    /* steps between admission points (0: 16) */
    void* stream;           /* cudaStream_t for all work (NULL: the server creates one) */
    size_t host_pinned_bytes; /* pinned host arena for request grids (0: none): a request
                               * placed there is uploaded and read back without staging,
                               * so the worker keeps the GPU fed; others use pageable memory */
} cfd_server_options;

typedef struct cfd_request_info {
    int state;              /* CFD_REQ_* */
    int error;
    int steps;              /* steps the solve took */
    double t;               /* its final simulated time */
    double submit_s;        /* submission time since server start */
    double queue_s;         /* submit -> admission */
    double run_s;           /* admission -> result on the host */
    double latency_s;       /* submit -> result on the host */
} cfd_request_info;

typedef struct cfd_server_stats {
    int64_t completed, admitted, queued, running, max_running, rounds;
    double cell_updates;    /* completed solves: cells x steps */
    double busy_s, wall_s;  /* worker time in step rounds; time since creation */
    double device_s;        /* CUDA-event time of the step rounds */
    size_t used_bytes, budget_bytes;
} cfd_server_stats;

typedef struct cfd_server cfd_server;
/* Creates a server and starts its worker thread.  No counterpart in the
 * reference, which runs one problem per process (sourcecode/main.cpp:17-48). */
int cfd_server_create(const cfd_server_options* opt, cfd_server** out);
/* Queues a solve of `steps` steps (or to cfg.T) from a ghosted AoS initial
 * grid, which is copied; CFD_ERR_BUDGET if it can never fit. */
int cfd_server_submit(cfd_server* s, const cfd_config* cfg, const double* ic, int steps,
                      int64_t* id);
/* Queues a solve whose initial condition is a seeded recipe, built on the
 * device at admission (no host grid is held while it waits). */
int cfd_server_submit_recipe(cfd_server* s, const cfd_config* cfg, int recipe, uint64_t seed,
                             int nbubbles, int steps, int64_t* id);
/* Waits up to timeout_s (< 0: forever) for a request; on completion fills
 * info and copies the final ghosted grid to `result` (may be NULL). */
int cfd_server_wait(cfd_server* s, int64_t id, double timeout_s, cfd_request_info* info,
                    double* result);
/* Forgets a finished request (frees its host copy). */
int cfd_server_release(cfd_server* s, int64_t id);
int cfd_server_get_stats(cfd_server* s, cfd_server_stats* st);
/* Stops the worker (in-flight solves are dropped) and frees everything. */
int cfd_server_destroy(cfd_server* s);

/* ---- test entry: the device flux of single faces -------------------------
 * flux_computation of the MUSCL-Hancock (or Godunov) solver
 * (headers/flux_solver_MUSCLhancock.hpp:128-227 / A: :272-376) evaluated on
 * the GPU for `nfaces` independent 4-cell (2-cell for Godunov) stencils of
 * conserved states, host arrays.  flux: nfaces*nvar, u_star and z_star:
 * nfaces each (z_star may be NULL for Euler). */
int cfd_face_flux(const cfd_config* cfg, int nfaces, const double* stencils, double dt,
                  double dx, double* flux, double* u_star, double* z_star);

#ifdef __cplusplus
}
#endif
#endif
