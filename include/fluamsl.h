/* fluamsl.h -- C ABI of libfluamsl, a B200 (sm_100a) implementation of
 * fluam's Stokes-limit immersed-boundary step ("Brownian dynamics without
 * Green's functions", the midpoint scheme of Delong et al., JCP 140, 134110,
 * 2014, Sec. IV.B).
 *
 * The reference path this library replaces is a set of process globals and
 * argument-less functions:
 *   bool schemeStokesLimit()     src/schemeStokesLimit.cu:27-98
 *   bool runSchemeStokesLimit()  src/runSchemeStokesLimit.cu:21-298
 *   main(argc, argv)             src/main.cpp:28-112 (loadDataMain + dispatch)
 * Here the state lives in an opaque handle.  All functions return 0 on
 * success and a negative FSL_E* code on failure (no exceptions cross the
 * boundary); fsl_last_error() gives a one-line message for the calling
 * thread.  The caller owns every host buffer; the handle owns every device
 * buffer.  A handle is used by one host thread at a time.
 *
 * Array layouts follow the reference: particle arrays are structure-of-arrays
 * x[0..np) | y[0..np) | z[0..np) in double precision (rxParticle, ...); fields
 * are component-major [3][nc] with cell index x + y mx + z mx my, and the
 * x component of cell i lives on the +x face of that cell.
 */
#ifndef FLUAMSL_H
#define FLUAMSL_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
enum {
  FSL_OK = 0,
  FSL_E_ARG = -1,        /* invalid argument or configuration            */
  FSL_E_CUDA = -2,       /* CUDA runtime error (message has the text)     */
  FSL_E_NOMEM = -3,      /* device allocation failed                      */
  FSL_E_KERNEL = -4,     /* a kernel raised its error word (see status)   */
  FSL_E_IO = -5,         /* file could not be read or written             */
  FSL_E_INPUT = -6       /* data.main keyword error (ERROR INPUT FILE)    */
};

/* ---- options that extend the reference ------------------------------- */
enum { FSL_PAIR_NONE = 0, FSL_PAIR_TABLE_LJ = 1, FSL_PAIR_SOFT = 2 };
enum { FSL_RFD_REFERENCE = 0, FSL_RFD_PAPER = 1 };
/* The integrator: the midpoint scheme of keyword stokesLimit
 * (src/runSchemeStokesLimit.cu:163-285) or the first-order scheme of keyword
 * stokesLimitFirstOrder (src/runSchemeStokesLimitFirstOrder.cu:163-241: one
 * solve per step with the RFD drift, the same predictor and corrector). */
/* The Gaussian-blob schemes of keywords quasi2D (RPY mobility of a blob in
 * a quasi-2-D geometry) and stokesLimit2D (2-D Stokes, optionally Saffman-
 * screened) on an mx x my grid (mz = 1): src/runSchemeQuasi2D.cu:20-260 with
 * src/quasi2DFunctions.cu.  FP64 throughout, as the reference. */
/* FSL_SCHEME_INCOMPRESSIBLE: the fluctuating incompressible Navier-Stokes
 * solver of keyword incompressible (src/runSchemeIncompressible.cu:20-155),
 * a fluid without particles (np = 0), FP64; its initial velocity is set by
 * fsl_set_velocity_f64. */
enum { FSL_SCHEME_MIDPOINT = 0, FSL_SCHEME_FIRST_ORDER = 1, FSL_SCHEME_QUASI2D = 2,
       FSL_SCHEME_STOKES2D = 3, FSL_SCHEME_INCOMPRESSIBLE = 4 };
/* Arithmetic of the fluid side (no counterpart in the reference, which is
 * FP64 throughout).  Particle positions, forces and the cell lists are FP64
 * in every form.
 *   FIXED64:      FP32 fields, noise and FFTs; spreading accumulated in 64-bit
 *                 fixed point (2^-40) with integer atomics: order-independent,
 *                 bit-reproducible run to run (the default);
 *   FLOAT_ATOMIC: the same with spreading accumulated by FP32 atomics (the
 *                 sum depends on the order the atomics land in);
 *   FP64:         noise, spreading (FP64 atomics), fields, FFTs and
 *                 interpolation all in FP64. */
enum { FSL_PRECISION_FIXED64 = 0, FSL_PRECISION_FLOAT_ATOMIC = 1, FSL_PRECISION_FP64 = 2 };

/* Bits of fsl_status.error_bits (device error word, sticky until cleared). */
enum {
  FSL_ERRBIT_FIXED_SAT = 1,   /* fixed-point spread value out of range      */
  FSL_ERRBIT_NONFINITE = 2,   /* non-finite force or position               */
  FSL_ERRBIT_GRID = 4         /* internal index check failed (access skipped) */
};

/* Configuration of one instance.  Field names follow data.main keywords
 * (src/loadDataMain.cu:173-683) where one exists. */
typedef struct fsl_config {
  int32_t mx, my, mz;            /* cells                                   */
  int32_t kernel;                /* Peskin kernel points: 3 (reference) or 4 */
  double lx, ly, lz;             /* celldimension                           */
  double shearviscosity;         /* eta                                     */
  double temperature;            /* kT                                      */
  double dt;
  double cutoff;                 /* pair cutoff rc (neighbour grid m=max(3,L/rc)) */
  double extra_mobility;         /* extraMobility (0 = off)                 */
  double soft_epsilon;           /* epsilon of U = eps (1 - r/rc)^2         */
  uint64_t seed;
  int32_t pair;                  /* FSL_PAIR_*; the reference is TABLE_LJ   */
  int32_t rfd;                   /* FSL_RFD_*                               */
  int32_t nonbonded;             /* computeNonBondedForces                  */
  int32_t device;                /* setDevice; -1 keeps the current device  */
  int32_t scheme;                /* FSL_SCHEME_*                            */
  int32_t precision;             /* FSL_PRECISION_*                         */
  /* quasi-2D family only (FSL_SCHEME_QUASI2D / FSL_SCHEME_STOKES2D) */
  int32_t ndrift;                /* nDrift (noise count only)               */
  int32_t use_rfd;               /* use_RFD: the thermal drift spread       */
  int32_t predictor_corrector;   /* predictorCorrector                      */
  /* 3-D Stokes schemes: 1 = accumulate fsl_observables in FP64 on the
   * device at the end of every step (one extra launch per step) */
  int32_t observables;
  double radius;                 /* hydrodynamicRadius                      */
  double saffman_kc;             /* saffmanCutOffWaveNumber (stokesLimit2D) */
  double saffman_width;          /* saffmanLayerWidth                       */
  double shear_amp;              /* viscosityMeasureAmplitude               */
  /* incompressible scheme only */
  double density;                /* densfluid                               */
} fsl_config;

typedef struct fsl_status {
  uint64_t step;                 /* steps taken since creation              */
  int32_t error_bits;            /* FSL_ERRBIT_*                            */
  int32_t np;
  int64_t nc;
  int32_t graph;                 /* 1 if steps replay a captured CUDA graph */
  int32_t launches_per_step;     /* kernels of this library in one step     */
} fsl_status;

/* Accumulated CUDA-event time of one stage of the step (profiling on). */
typedef struct fsl_stage_time {
  char name[32];
  int64_t launches;
  double total_ms;
} fsl_stage_time;

typedef struct fsl_handle fsl_handle;

/* Fill cfg with the reference's defaults (src/loadDataMain.cu:175-299) plus
 * kernel 3, TABLE_LJ, reference RFD.  Replaces nothing; convenience. */
void fsl_config_defaults(fsl_config* cfg);

/* Create an instance and upload np positions (SoA, double).  Replaces the
 * set-up half of schemeStokesLimit (src/schemeStokesLimit.cu:30-58:
 * createCells, createCellsStokesLimitGPU, createBoundariesRK2GPU). */
int fsl_create(const fsl_config* cfg, int64_t np, const double* q, fsl_handle** out);

/* Harmonic bonds and fixed-point tethers, in the reference's file order
 * (src/initializeBondedForces.cpp:31-170, src/createBondedForcesGPU.cu:21-133).
 * fxyz holds 3 doubles per tether. */
int fsl_load_bonds(fsl_handle* h, int64_t nbonds, const int32_t* bi, const int32_t* bj,
                   const double* k, const double* r0, int64_t nfixed, const int32_t* fi,
                   const double* fk, const double* fr0, const double* fxyz);

/* Directed bond entries, as the reference holds them in memory and as the
 * old bond-file format (bondedForcesVersion 1) lists them: entry b adds the
 * spring (k[b], r0[b]) towards particle bj[b] to the force on bi[b] only, so
 * a bond appears once from each end (src/initializeBondedForcesOldVersion.cpp:
 * 41-238; the reference's CSR bondsParticleParticle/Offset,
 * bondsIndexParticleParticle, kSpring/r0ParticleParticle of
 * src/initializeBondedForces.cpp:31-170 expands to these entries).  Entries
 * are grouped by bi in their order.  Tethers as fsl_load_bonds. */
int fsl_load_bonds_directed(fsl_handle* h, int64_t nentries, const int32_t* bi, const int32_t* bj,
                            const double* k, const double* r0, int64_t nfixed, const int32_t* fi,
                            const double* fk, const double* fr0, const double* fxyz);

/* Advance nsteps midpoint steps (the body of the loop in
 * src/runSchemeStokesLimit.cu:163-285).  Runs on the handle's stream; returns
 * after the work is queued unless an error check needs the device. */
int fsl_step(fsl_handle* h, int64_t nsteps);

/* Block until queued work is done and read the device error word. */
int fsl_sync(fsl_handle* h);

/* Particle positions q^n (gpuToHostStokesLimit, src/gpuToHostStokesLimit.cu:36-38). */
int fsl_get_positions(fsl_handle* h, double* out);
int fsl_set_positions(fsl_handle* h, const double* in);
/* One step with its positions in and out: fsl_set_positions(in),
 * fsl_step(1), fsl_get_positions(out) with the same results, bit for bit
 * (in may equal out).  With page-locked host buffers both copies are nodes
 * of the step's CUDA graph and the copy in runs beside the step's noise,
 * which reads no position; the graph is kept for the same pair of buffers,
 * and a plain fsl_step in between captures it again.  Pageable buffers
 * take the three calls.  The reference moves positions between host and
 * device around its step loop (src/runSchemeStokesLimit.cu:163-285,
 * src/gpuToHostStokesLimit.cu). */
int fsl_step_io(fsl_handle* h, const double* in, double* out);
/* Particle forces F^{n+1/2} of the last step: what the reference writes to
 * <out>.velocityParticles (src/gpuToHostStokesLimit.cu:41-43). */
int fsl_get_forces(fsl_handle* h, double* out);
/* Fluid velocity of the last solve, float [3][nc] (not written by the
 * reference on this path; exposed for checks). */
int fsl_get_velocity(fsl_handle* h, float* out);
/* The same as double [3][nc], in every precision form (the only full-precision
 * read of the FP64 form's field). */
int fsl_get_velocity_f64(fsl_handle* h, double* out);
/* Incompressible scheme: upload the staggered velocity double [3][nc] and
 * project it onto divergence-free fields, as the scheme does before its
 * first step (src/runSchemeIncompressible.cu:82-96). */
int fsl_set_velocity_f64(fsl_handle* h, const double* in);
int fsl_get_status(fsl_handle* h, fsl_status* st);
/* The autotuner's picks for this instance (fsl_class_tuning, below). */
struct fsl_class_tuning;
int fsl_get_tuning(fsl_handle* h, struct fsl_class_tuning* out);

/* FP64 accumulators kept on the device when fsl_config.observables is 1
 * (3-D Stokes schemes).  No counterpart in the reference, which computes no
 * observables on this path.  q0 are the reference positions: the positions
 * given to fsl_create, or those at the last fsl_reset_observables. */
typedef struct fsl_observables {
  int64_t steps;                 /* steps accumulated since q0 was set        */
  double msd;                    /* (1/np) sum_i |q_i - q0_i|^2 after the last step */
  double msd_sum;                /* sum of msd over the accumulated steps     */
  double displacement[3];        /* (1/np) sum_i (q_i - q0_i): centre-of-mass drift */
  double force[3];               /* sum_i F_i of the step's last force evaluation */
  double momentum[3];            /* sum over cells of v dV of the last solve (the
                                    fluid momentum per unit density)         */
  double momentum_sum[3];        /* sum of momentum over the accumulated steps */
} fsl_observables;
/* Read the accumulators (waits for the handle's queued work). */
int fsl_get_observables(fsl_handle* h, fsl_observables* out);
/* q0 := the current positions; accumulators := 0 (queued on the stream). */
int fsl_reset_observables(fsl_handle* h);

int fsl_set_step(fsl_handle* h, uint64_t step);
/* Clears the error word.  It also clears the cell-list counters and the grid
 * barrier of the single-launch list build and requests fresh lists at the
 * next force evaluation, so an instance whose list build gave up
 * (FSL_ERRBIT_GRID: the build is skipped until the bit is cleared) steps
 * normally again afterwards. */
int fsl_clear_errors(fsl_handle* h);
/* Capture one step into a CUDA graph and replay it from then on (on by
 * default once the first step has run; 0 turns it off). */
int fsl_set_graph(fsl_handle* h, int enable);
/* The handle's CUDA stream (cudaStream_t), for callers that order work. */
void* fsl_stream(fsl_handle* h);
/* Per-stage timing with CUDA events recorded on the handle's stream between
 * the stages of every step (captured into the graph as well).  While it is
 * on, fsl_step waits for each step to finish.  fsl_profile(h, 1) also clears
 * the accumulated times.  The reference only times the whole run
 * (src/saveTime.cpp:24-45). */
int fsl_profile(fsl_handle* h, int enable);
int fsl_profile_read(fsl_handle* h, fsl_stage_time* out, int32_t max, int32_t* n);
void fsl_destroy(fsl_handle* h);
const char* fsl_last_error(void);

/* ---- drop-in driver ---------------------------------------------------- */
/* Run a whole fluam Stokes-limit job from a data.main file: the same
 * keywords, the same output files (<outputname>.data.main, .cuda, .seed,
 * .time, .particles, .velocityParticles).  Mirrors main() + schemeStokesLimit()
 * (src/main.cpp:28-112, src/schemeStokesLimit.cu:27-98).  Returns 0 on
 * success. */
int fsl_run_data_main(const char* path);
/* Parse a data.main into cfg and the run controls without touching a GPU
 * (src/loadDataMain.cu:173-683).  numsteps/samplefreq/relax may be NULL. */
int fsl_parse_data_main(const char* path, fsl_config* cfg, int64_t* numsteps,
                        int64_t* samplefreq, int64_t* relax, int64_t* np);

/* ---- fluid output (opt-in; the reference's Stokes path writes none) ------
 * v is the staggered fluid velocity [3][mz][my][mx] (x fastest), e.g. from
 * fsl_get_velocity_f64.  The drop-in driver calls these for the reference's
 * keywords saveFluid 1 and saveVTK 1 (with savefreq). */
/* <out>.fluidFinalConfiguration in the text format of
 * saveFluidFinalConfiguration (src/saveFluidFinalConfiguration.cu:30-75):
 * header, then per cell the density and the staggered velocity. */
int fsl_write_fluid_final(const char* path, const fsl_config* cfg, double density,
                          const double* pressure3, int32_t thermostat, const double* v);
/* Legacy ASCII VTK rectilinear grid of (mx+1) x (my+1) x (mz+1) nodes with the
 * cell-centred velocity as CELL_DATA, in the layout of the reference's VTK
 * writer (src/saveFluidVTK.cu:33-250 via src/visit_writer.c:321-460,899-1015). */
int fsl_write_fluid_vtk(const char* path, int32_t mx, int32_t my, int32_t mz, const double* v);

/* ---- component entry points (one stage of the step each) --------------- */
/* Non-bonded cell list at the current positions: cell of each particle, the
 * start offset of every neighbour-grid cell (mN+1 entries) and the particle
 * indices sorted by cell, ascending inside a cell.  Replaces
 * findNeighborParticlesStokesLimit_1 (src/stokesLimitFunctions.cu:23-61). */
int fsl_neighbor_grid(fsl_handle* h, int32_t* dims3);
int fsl_cell_list(fsl_handle* h, int32_t* cell_of, int32_t* start, int32_t* sorted);
/* Forces at the current positions (pair + bonded), the force half of
 * kernelSpreadParticlesForceStokesLimit (src/stokesLimitFunctions.cu:83-657). */
int fsl_compute_forces(fsl_handle* h, double* F);
/* f = S(q) F / dV at the current positions for given particle forces F
 * (spread + addSpreadedForcesStokesLimit, src/stokesLimitFunctions.cu:659-1681). */
int fsl_spread(fsl_handle* h, const double* F, double* f);
/* v = (eta L)^-1 P W for a given real field W [3][nc] (FFT, kernelShift,
 * kernelUpdateVstokesLimit, inverse FFT, normalisation:
 * src/runSchemeStokesLimit.cu:198-214). */
int fsl_solve(fsl_handle* h, const double* W, double* v);
/* u = J(q) v at the current positions for a given field v [3][nc]
 * (src/stokesLimitFunctions.cu:2616-2642). */
int fsl_interpolate(fsl_handle* h, const double* v, double* u);
/* Noise array entries [first, first+count) of draw t, as floats. */
int fsl_noise(fsl_handle* h, uint64_t t, uint64_t first, int64_t count, float* out);

/* ---- batched instances --------------------------------------------------
 * No counterpart in the reference, which runs one instance per process
 * (process globals, src/schemeStokesLimit.cu:27-98).  A batch holds n
 * independent instances, each with its own configuration, particles, seed
 * and step counter.  Instances with the same cells, neighbour-grid extents
 * (max(3, int(L/cutoff)) per direction) and kernel width form a size class:
 * one kernel launch per stage serves a whole class, the classes run on
 * separate streams, and from the second step on a step of the batch is one
 * CUDA graph launch.  Each instance's results are bit-identical to the same
 * instance run alone through fsl_create/fsl_step.  Instance i is addressed
 * by its index in the arrays given to fsl_batch_create.  Packed particle
 * arrays concatenate the instances' SoA blocks (3 np_i doubles each) in
 * index order. */
typedef struct fsl_batch fsl_batch;

typedef struct fsl_batch_info {
  int32_t n;                     /* instances                                 */
  int32_t classes;               /* size classes (launch groups)              */
  int32_t graph;                 /* 1 if steps replay a captured CUDA graph   */
  int32_t launches_per_step;     /* kernels of this library in one step       */
  int64_t np_total;              /* particles over all instances              */
  int64_t nc_total;              /* cells over all instances                  */
  int64_t device_bytes;          /* device memory held by the batch           */
} fsl_batch_info;

/* cfgs[i], np[i] and q[i] (SoA, 3 np[i] doubles) describe instance i; all
 * instances live on one device (the first cfgs[i].device >= 0, else the
 * current one). */
int fsl_batch_create(int32_t n, const fsl_config* cfgs, const int64_t* np, const double* const* q,
                     fsl_batch** out);
int fsl_batch_load_bonds(fsl_batch* b, int32_t i, int64_t nbonds, const int32_t* bi,
                         const int32_t* bj, const double* k, const double* r0, int64_t nfixed,
                         const int32_t* fi, const double* fk, const double* fr0, const double* fxyz);
int fsl_batch_step(fsl_batch* b, int64_t nsteps);
/* Block until queued work is done; FSL_E_KERNEL if any instance's error word
 * is set (the message names the first such instance). */
int fsl_batch_sync(fsl_batch* b);
int fsl_batch_get_positions(fsl_batch* b, int32_t i, double* out);
int fsl_batch_get_forces(fsl_batch* b, int32_t i, double* out);
int fsl_batch_get_status(fsl_batch* b, int32_t i, fsl_status* st);
/* fsl_get_observables / fsl_reset_observables of instance i. */
int fsl_batch_get_observables(fsl_batch* b, int32_t i, fsl_observables* out);
int fsl_batch_reset_observables(fsl_batch* b, int32_t i);
/* All instances' positions in one packed array (one copy each way plus one
 * gather/scatter kernel). */
int fsl_batch_get_positions_packed(fsl_batch* b, double* out);
int fsl_batch_set_positions_packed(fsl_batch* b, const double* in);
/* The same, asynchronous on the batch's stream: `host` must stay valid (and,
 * for a copy that overlaps other work, be page-locked) until the stream
 * reaches the copy. */
int fsl_batch_get_positions_packed_async(fsl_batch* b, double* host);
int fsl_batch_set_positions_packed_async(fsl_batch* b, const double* host);
/* One step of every instance with all positions in and out in the packed
 * layout: fsl_batch_set_positions_packed(in), fsl_batch_step(1),
 * fsl_batch_get_positions_packed(out) with the same results, bit for bit
 * (in may equal out).  With page-locked host buffers the copies and the
 * scatter and gather kernels are nodes of the step's CUDA graph: the copy
 * in and the scatter on a stream of their own beside every size class's
 * noise, the gather and the copy out after the join; the graph is kept
 * while the same pair of buffers comes back.  Pageable buffers take the
 * three calls. */
int fsl_batch_step_io(fsl_batch* b, const double* in, double* out);
int fsl_batch_set_graph(fsl_batch* b, int enable);
int fsl_batch_get_info(fsl_batch* b, fsl_batch_info* info);

/* What the autotuner of one size class picked and measured.  A class (the
 * instances with the same cells, kernel, scheme and precision) is tuned at
 * its first step outside graph capture: the z-pass tile of the transform,
 * the planes per block of its plane passes, the transform schedule, and for
 * a batch of small instances the list build.  Every choice computes the same bits, so the picks change speed
 * only.  No counterpart in the reference, whose launch shape is a fixed
 * heuristic on the particle count (src/runSchemeStokesLimit.cu:24-68). */
typedef struct fsl_class_tuning {
  int32_t mx, my, mz;            /* cells                                      */
  int32_t kernel;                /* 3- or 4-point                              */
  int32_t precision;             /* FSL_PRECISION_*                            */
  int32_t scheme;                /* FSL_SCHEME_*                               */
  int32_t n;                     /* instances in the class                     */
  int32_t tuned;                 /* 1 once the class's first step has run      */
  int32_t fft_schedule;          /* 0 plane passes, 1 five passes, -1 other    */
  int32_t z_tile_kx, z_tile_ky;  /* z-pass tile picked (0: no register z pass) */
  int32_t z_threads;             /* threads per block of that tile             */
  int32_t z_candidates;          /* z tiles timed (at most 8)                  */
  float z_us[8];                 /* us per z-pass launch of each candidate     */
  float schedule_us[2];          /* us per transform: plane, five passes
                                    (0: not timed)                             */
  int32_t list_build;            /* 0 separate kernels, 1 one block per
                                    instance, 2 cooperative single launch,
                                    -1 no particles                            */
  float list_us[2];              /* us per build: separate, block per
                                    instance (0: not timed)                    */
  int32_t plane_pb;              /* planes per block of the plane passes
                                    picked (0: no register plane passes)       */
  int32_t plane_candidates;      /* planes-per-block candidates (at most 4)    */
  float plane_us[4];             /* us per plane-schedule transform of each
                                    candidate (0: not timed)                   */
} fsl_class_tuning;

/* Size class k of the batch, 0 <= k < fsl_batch_info.classes. */
int fsl_batch_get_class_tuning(fsl_batch* b, int32_t k, fsl_class_tuning* out);
void* fsl_batch_stream(fsl_batch* b);
void fsl_batch_destroy(fsl_batch* b);

/* ---- serving loop ---------------------------------------------------------
 * No counterpart in the reference (one instance per process run to
 * completion).  A server owns one device and a scheduler thread.  Requests
 * (a configuration, positions and a step count) are queued by
 * fsl_server_submit from any thread.  The scheduler admits queued requests
 * in arrival order into slots of their size class while the device memory of
 * all slots stays within the budget, and advances every admitted request
 * together: one launch per stage and size class, the whole step one CUDA
 * graph.  Requests that arrive while others run join at the next round; a
 * round lasts as many steps as the nearest completion (at most
 * max_round_steps), so every request takes exactly its own step count and
 * its results are bit-identical to the same instance run alone through
 * fsl_create/fsl_step.  Instance state stays on the device from admission to
 * completion; the slot of a finished request is reused by the next one of
 * its class.  All fsl_server_* calls are thread-safe. */
typedef struct fsl_server fsl_server;

typedef struct fsl_server_config {
  int64_t hbm_budget;            /* device bytes for instance state          */
  int32_t device;                /* -1 keeps the current device              */
  int32_t max_round_steps;       /* longest stretch between admissions       */
} fsl_server_config;

enum { FSL_REQ_QUEUED = 0, FSL_REQ_RUNNING = 1, FSL_REQ_DONE = 2, FSL_REQ_FAILED = 3 };

typedef struct fsl_request_info {
  int32_t state;                 /* FSL_REQ_*                                 */
  int32_t error_bits;            /* FSL_ERRBIT_* of the instance              */
  int64_t np;
  int64_t steps;                 /* requested                                 */
  int64_t steps_done;
  double submit_s, start_s, done_s;  /* on the server's clock (seconds)       */
} fsl_request_info;

typedef struct fsl_server_stats {
  int64_t submitted, completed, failed, queued, running;
  int64_t rounds, steps, particle_steps;  /* steps: sum over requests        */
  int64_t bytes_held, slots;
  int64_t groups, captures;
  double busy_s;                 /* time the scheduler spent in rounds        */
  double now_s;                  /* the server's clock                        */
} fsl_server_stats;

void fsl_server_config_defaults(fsl_server_config* cfg);
int fsl_server_create(const fsl_server_config* cfg, fsl_server** out);
/* Copies q (SoA, 3 np doubles); *id identifies the request. */
int fsl_server_submit(fsl_server* s, const fsl_config* cfg, int64_t np, const double* q,
                      int64_t nsteps, int64_t* id);
int fsl_server_poll(fsl_server* s, int64_t id, fsl_request_info* info);
/* Blocks until the request is done or failed, or timeout_s elapses
 * (negative: no limit); returns FSL_OK either way, with the state in info. */
int fsl_server_wait(fsl_server* s, int64_t id, double timeout_s, fsl_request_info* info);
/* Final positions and forces (F^{n+1/2} of the last step) of a finished
 * request, then forgets it.  Either output may be NULL. */
int fsl_server_result(fsl_server* s, int64_t id, double* q_out, double* F_out);
int fsl_server_get_stats(fsl_server* s, fsl_server_stats* st);
/* Stops the scheduler after its current round; unfinished requests fail. */
void fsl_server_destroy(fsl_server* s);

/* ---- cell list without device allocation -------------------------------
 * No counterpart in the reference.  The same cell list as fsl_cell_list, for
 * callers that must not allocate device memory: frameworks that own all
 * device memory through their own pool, and loops that keep other GPU work
 * in flight (cudaMalloc/cudaFree can synchronise the whole device).  It takes
 * no handle.  q_dev (np x 3 doubles, SoA), cell_of_dev (np), start_dev (m+1,
 * m = neighbour-grid cells of max(3, int(L/cutoff)) per direction) and
 * sorted_dev (np) are device memory owned by the caller; the work is queued
 * on `stream` (a cudaStream_t, NULL for the default stream).  The sort's
 * scratch is a fixed array inside the library (about 9 MiB on every GPU that
 * loads it, held until exit), which limits a call to 262,144 particles and
 * 1,048,576 neighbour-grid cells; larger sizes are rejected with FSL_E_ARG.
 * The first call on a device looks up that array's address, so make the first
 * call on each device before any stream capture.  All calls share the array:
 * calls whose work overlaps on the GPU (different streams, or different host
 * threads on one device) race and must be ordered by the caller.  A
 * non-finite coordinate gives that particle an arbitrary in-range cell and is
 * not reported here. */
int fsl_cell_list_noalloc(double lx, double ly, double lz, double cutoff, int64_t np,
                          const double* q_dev, int32_t* cell_of_dev, int32_t* start_dev,
                          int32_t* sorted_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FLUAMSL_H */
