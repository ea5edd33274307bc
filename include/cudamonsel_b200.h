/*
 * cudamonsel_b200.h -- C ABI of the B200 electron-transport engine.
 *
 * The engine replaces the CPU trajectory loop of CudaMONSEL
 * (NISTMonte/MonteCarloSS.cu:107-231 and everything it calls) with CUDA
 * kernels for sm_100a.  A caller describes the same objects the reference's
 * C++ API builds -- SEmaterial, MONSEL_MaterialScatterModel and its
 * ScatterMechanism / SlowingDownAlg / BarrierScatterMechanism plug-ins,
 * NormalShapes, the Region tree, the GaussianBeam and BackscatterStats -- and
 * then runs trajectories for a list of beam landing points (pixels).
 *
 * Conventions
 *   - Units are the reference's: SI (J, m, m^2, kg/m^3).
 *   - Every function returns 0 on success and a negative CM_E* code on error;
 *     cm_last_error() then describes the failure (thread-local).
 *   - Object handles are small non-negative ints returned through out-params.
 *   - Pointers are host pointers unless the name says _device.
 *   - A context is not thread-safe; use one per host thread.
 *
 * Reference paths below are relative to CudaMONSEL/CudaMONSEL/gov/nist/.
 */
#ifndef CUDAMONSEL_B200_H
#define CUDAMONSEL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CM_OK 0
#define CM_EINVAL -1    /* bad argument or handle */
#define CM_ECUDA -2     /* CUDA runtime error */
#define CM_ENOMEM -3    /* device allocation failed */
#define CM_ESTATE -4    /* scene incomplete or inconsistent */
#define CM_EOVERFLOW -5 /* a device queue overflowed (secondary pool too small) */
#define CM_ELIMIT -6    /* iteration limit reached before all trajectories ended */
#define CM_ECANCELED -7 /* the job was cancelled */
#define CM_ETIMEOUT -8  /* a bounded wait on the device ran out (a table copy into shared memory did not land) */

#define CM_PREC_FP64 0  /* plain form: all transport arithmetic in double */
#define CM_PREC_FP32 1  /* batched form: float physics, double positions and plane solves */

#define CM_OPT_JMONSEL_FIXES 1 /* refraction at barriers, d3 abscissae; default is the reference as written */
#define CM_OPT_EXACT_CSG 2     /* FP32 too walks NormalIntersectionShape trees as the reference does; by default
                                  FP32 merges intersections of plane sets into single plane sets */
#define CM_OPT_SCAN_CHILDREN 4 /* test every child of a region in order, as RegionBase does; by default a region
                                  with many children finds them through an x-y grid (same results) */
#define CM_OPT_GLOBAL_TABLES 16 /* kernels read every table from global memory (through L1/L2); by default the small
                                   tables are staged into each block's shared memory by a bulk copy (same results) */
#define CM_OPT_QUEUE_STEPS 8   /* one step per iteration through the queue kernels to the end of a run; by default
                                  the tail of a run (fewer electrons left than fill the GPU) takes several whole
                                  steps per thread (same results) */

typedef struct cm_context cm_context;

/* ---- context -------------------------------------------------------------- */
int cm_context_create(int device, cm_context** out);
int cm_context_destroy(cm_context* ctx);
/* forgets the scene (materials, models, tables, shapes, regions, options) so the context can describe another */
int cm_context_reset(cm_context* ctx);
const char* cm_last_error(void);
int cm_set_options(cm_context* ctx, int options);

/* Launch settings of the transport loop (no reference counterpart: the reference runs one trajectory at a
 * time), one set per precision.  0 = the built-in default.  Every setting gives the same tallies, because
 * each electron's random stream is keyed by its lineage, so they change only the speed. */
typedef struct {
  int wave;                    /* electrons per wave segment (default 2^21; 1024 .. 2^24) */
  int tail_below;              /* k_steps runs the tail once fewer electrons are left (default 262144) */
  int tail_steps;              /* whole steps per thread and launch in the tail (default 32) */
  int blocks_per_sm;           /* grid = SMs x blocks_per_sm blocks of 256 threads (default 8) */
  double ms;                   /* cm_autotune: device time of the transport loop under these settings */
  int pool;                    /* secondary-pool records per wave electron (default by the highest beam
                                  energy: 8 at 1 keV and below, 8 per keV above, up to 64; 1 .. 64); a run
                                  that overflows the pool is run again with twice the pool */
} cm_tuning;
int cm_get_tuning(cm_context* ctx, int precision, cm_tuning* out);
int cm_set_tuning(cm_context* ctx, int precision, const cm_tuning* tuning);
int cm_version(void);
/* The directory of the data files the library ships (NistXSec/E%02d.bin: NIST SRD-64 elastic tables):
 * $CM_DATA_DIR, else the "data" folder beside the loaded libcudamonsel_b200.so.  No reference counterpart
 * (the reference opens its data by paths relative to the working directory). */
const char* cm_data_dir(void);

/* ---- data ------------------------------------------------------------------- */
/* NIST SRD-64 elastic table of one element, as NISTMottScatteringAngle::loadData
 * reads it (EPQLibrary/NISTMottScatteringAngle.cu:44-66): 61 cross sections in
 * Bohr radii squared, then 61 x 201 quantiles (row = energy node). */
int cm_add_mott_element(cm_context* ctx, int Z, const double* spwem61, const double* x1_61x201);
/* A NUTableInterpolation table (JMONSEL/NUTableInterpolation.cu:117-228):
 * dim in 1..3, n[dim] grid sizes, the axes concatenated, values last index fastest. */
int cm_add_table(cm_context* ctx, int dim, const int* n, const double* axes, const double* values, int* out_table);

/* ---- materials and scatter models ---------------------------------------- */
/* SEmaterial (JMONSEL/SEmaterial.cu) with its Composition: nel elements given by
 * Z, atomic weight (g/mol) and normalized weight fraction.  nel = 0 is vacuum. */
int cm_add_material(cm_context* ctx, int nel, const int* Z, const double* atomic_weight, const double* weight_fraction,
                    double density, double workfunction, double energy_cb_bottom, double bandgap, int ncore,
                    const double* core_energies, int* out_material);
/* MONSEL_MaterialScatterModel(mat, ExpQMBarrierSM(mat)) (JMONSEL/MONSEL_MaterialScatterModel.cu:13-37) */
int cm_add_msm(cm_context* ctx, int material, int* out_msm);
/* SelectableElasticSM(mat, NISTMottRS factory) (JMONSEL/SelectableElasticSM.cu:10-18).  method 1 =
 * NISTMottRS::Factory (Browning-scaled below 50 eV), 2 = Factory100 (Browning-scaled below 100 eV),
 * 3 = Factory100Lin (cross section linear in energy below 100 eV); JMONSEL/NISTMottRS.cu:76-119, :506-512 */
int cm_msm_add_nistmott(cm_context* ctx, int msm, int method, int* out_mech);
/* TabulatedInelasticSM(mat, methodSE, tables, energyOffset) (JMONSEL/TabulatedInelasticSM.cu:23-66);
 * tables = {IIMFP, reduced deltaE, theta, SE E0} */
int cm_msm_add_tabulated(cm_context* ctx, int msm, int method_se, double energy_offset, const int tables[4], int* out_mech);
/* FittedInelSM(mat, energySEgen, JoyLuoNieminenCSD(mat, breakE)) (JMONSEL/FittedInelSM.cu:8-11) */
int cm_msm_add_fitted(cm_context* ctx, int msm, double energy_se_gen, double break_e, int* out_mech);
/* GanachaudMokraniPhononInelasticSM (JMONSEL/GanachaudMokraniPhononInelasticSM.cu:8-17) */
int cm_msm_add_phonon(cm_context* ctx, int msm, double ratemult, double phonon_e, double temperature, double eps0,
                      double eps_infinity, int* out_mech);
/* GanachaudMokraniPolaronTrapSM (JMONSEL/GanachaudMokraniPolaronTrapSM.cu:8-12) */
int cm_msm_add_polaron(cm_context* ctx, int msm, double prefactor, double extinction, int* out_mech);
/* MONSEL_MaterialScatterModel::setCSD(JoyLuoNieminenCSD(mat, breakE)) (MONSEL_MaterialScatterModel.cu:146-152) */
int cm_msm_set_csd_jln(cm_context* ctx, int msm, double break_e);
/* MONSEL_MaterialScatterModel::setMinEforTracking */
int cm_msm_set_min_e(cm_context* ctx, int msm, double min_e);
/* ExpQMBarrierSM(mat) classical (1) or ExpQMBarrierSM(mat, lambda) (0) (JMONSEL/ExpQMBarrierSM.cu:12-28) */
int cm_msm_set_barrier(cm_context* ctx, int msm, int classical, double lambda);

/* ---- shapes and regions ------------------------------------------------------ */
int cm_shape_sphere(cm_context* ctx, const double center[3], double radius, int* out_shape);   /* NISTMonte/Sphere.cu */
/* NormalMultiPlaneShape with n planes (normal, point) (JMONSEL/NormalMultiPlaneShape.cu) */
int cm_shape_planes(cm_context* ctx, int n, const double* normals, const double* points, int* out_shape);
int cm_shape_intersection(cm_context* ctx, int a, int b, int* out_shape); /* JMONSEL/NormalIntersectionShape.cu */
/* NormalUnionShape(a, b) (JMONSEL/NormalUnionShape.cu) */
int cm_shape_union(cm_context* ctx, int a, int b, int* out_shape);
/* NormalCylindricalShape(end0, end1, radius) (JMONSEL/NormalCylindricalShape.cu).  As compiled, the
 * reference normalises the axis by a length it has not initialised yet (read as 0), so the cylinder is
 * never struck by a step; that is reproduced unless CM_OPT_JMONSEL_FIXES is set when it is created. */
int cm_shape_cylinder(cm_context* ctx, const double end0[3], const double end1[3], double radius, int* out_shape);
int cm_shape_translate(cm_context* ctx, int shape, const double distance[3]);
/* ITransform::rotate(pivot, phi, theta, psi): Euler angles phi about z, theta about y, psi about z, around
 * pivot (Utility/Transform3D.cu:5-128), for NormalMultiPlaneShape (NormalMultiPlaneShape.cu:257-261: every
 * plane's normal and point), NormalCylindricalShape (NormalCylindricalShape.cu:324-330: its end, its axis
 * and the axis normalised by the length it was built with, so a rotation also normalises the axis of a
 * cylinder built without CM_OPT_JMONSEL_FIXES) and Sphere; intersections and unions rotate their parts. */
int cm_shape_rotate(cm_context* ctx, int shape, const double pivot[3], double phi, double theta, double psi);
/* NShapes::createLine(topz, width, length, thetal, thetar, radl, radr) (JMONSEL/NShapes.cu:55-149); a corner
 * radius adds a clipping plane and a cylinder joined by a union.  The reference's left corner uses the right
 * sidewall (NShapes.cu:140); CM_OPT_JMONSEL_FIXES set when the line is created uses the left one. */
int cm_shape_line(cm_context* ctx, double topz, double width, double length, double thetal, double thetar, double radl,
                  double radr, int* out_shape);
/* Region(parent, msm, shape) (NISTMonte/RegionBase.cu:193-200); parent -1 makes the chamber */
int cm_region_add(cm_context* ctx, int parent, int msm, int shape, int* out_region);

/* ---- trajectories ---------------------------------------------------------- */
/* One run: for each pixel p, pixel_nprim[p] trajectories from a GaussianBeam of
 * width beam_width centred at pixel_center[3p..3p+2] with energy pixel_energy[p],
 * each tallied by a BackscatterStats(monte, pixel_nbins[p]) attached for that
 * pixel (NISTMonte/BackscatterStats.cu:107-181). */
typedef struct {
  int chamber;                 /* region handle of the chamber */
  int precision;               /* CM_PREC_FP64 or CM_PREC_FP32 */
  int npix;
  double beam_width;           /* m (Gaussian sigma) */
  const double* pixel_center;  /* [3*npix] m */
  const double* pixel_energy;  /* [npix] J */
  const int* pixel_nprim;      /* [npix] */
  const int* pixel_nbins;      /* [npix], 1..1024 */
  uint64_t seed;
  int hist_stride;             /* >= max(pixel_nbins) + 2 */
  int wave;                    /* electrons per wave; 0 = the context's cm_tuning.wave, else the default;
                                  at most 2^27 (CM_EINVAL beyond).  Run buffers that do not fit in the
                                  device's free memory: CM_ENOMEM, nothing allocated, the context usable. */
  int max_iterations;          /* 0 = default */
  const uint64_t* pixel_key;   /* [npix] random-stream key of each pixel, or NULL: derived from seed and index.
                                  A pixel's result depends only on its key, its beam and primary count,
                                  not on the other pixels of the run. */
  int profile;                 /* nonzero: time each kernel with CUDA events inside the loop */
  /* BackscatterStats' elevation and azimuthal histograms (NISTMonte/BackscatterStats.cu:105-106,147-165:
   * Histogram(0, pi, 180) of pi/2 - atan2(z, r) and Histogram(0, 2 pi, 360) of atan2(y, x) at the escape
   * point), per pixel, or NULL: [npix * CM_ELEVATION_COUNTS] and [npix * CM_AZIMUTH_COUNTS] counts, index =
   * bin + 1 as for back/fwd.  Every escape is counted, also those past the energy histogram's overflow slot.
   * Host arrays for cm_run, device arrays for cm_run_device; not taken by cm_run_noalloc or the job server. */
  uint32_t* elevation;
  uint32_t* azimuth;
  /* BackscatterStats' detected-electron log (setLogDetected, BackscatterStats.cu:166-168), or NULL: the first
   * escape_log_cap escapes in arrival order (which varies from run to run); the run's stats.escapes says how
   * many there were.  Host array for cm_run, device array for cm_run_device. */
  struct cm_escape_record* escape_log;
  int64_t escape_log_cap;
  /* [npix] index of each pixel's first primary, or NULL: 0.  Primary k of a pixel draws from a stream keyed
   * by (pixel key, k), so a scan can run in parts -- pixel_first = primaries done so far, pixel_nprim = the
   * next part -- and the parts' tallies add up to exactly those of one run: checkpoint/resume of a scan from
   * (pixel_first, tallies).  Host array for cm_run, device array for cm_run_device; not taken by
   * cm_run_noalloc or the job server (CM_EINVAL). */
  const int64_t* pixel_first;
} cm_run_desc;

#define CM_ELEVATION_COUNTS 182 /* 180 bins + underflow + overflow */
#define CM_AZIMUTH_COUNTS 362   /* 360 bins + underflow + overflow */

/* BackscatterStats::Datum (BackscatterStats.cu:10-57): the electron, its step count, kinetic energy, position
 * and direction angles when it left the chamber.  The electron is named by its random-stream key (the
 * reference numbers electrons in creation order, which a parallel run does not have). */
typedef struct cm_escape_record {
  uint64_t electron;
  int32_t pixel;
  int32_t step;
  double energy_eV;
  double position[3];          /* m */
  double theta, phi;           /* direction (cos phi sin theta, sin phi sin theta, cos theta) */
} cm_escape_record;

/* kernels of one wavefront iteration, in launch order */
#define CM_K_FLIGHT 0
#define CM_K_ELASTIC 1
#define CM_K_INELASTIC 2
#define CM_K_MISC 3
#define CM_K_SPAWN 4
#define CM_K_TAIL 5

typedef struct {
  int64_t primaries, steps, scatter_events, barrier_events, escapes, secondaries, iterations;
  double device_ms;            /* time of the transport loop on the device */
  double kernel_ms[6];         /* per kernel, summed over launches (profile != 0 only) */
  int64_t kernel_launches[6];
  int64_t units[4];            /* electrons handled by flight, elastic, inelastic, misc */
  int64_t step_launches;       /* launches of the several-steps-per-thread kernel that runs the tail of a
                                  run (when fewer electrons are left than fill the GPU); the queue kernels
                                  flight .. misc do not run in those iterations */
  int64_t step_units;          /* electrons those launches started with */
  double step_ms;              /* their time (profile != 0 only) */
  int64_t ended_zero_energy;   /* electrons with no energy left, in a region without scatter mechanisms,
                                  ended after 4096 steps (each one only bounces between barriers) */
  int64_t ended_step_limit;    /* electrons ended by the reference's 10^6-step limit
                                  (MONSEL_MaterialScatterModel.cu:86-90) */
  int64_t pool_restarts;       /* times the run (a job: its batch) overflowed the secondary pool and was
                                  run again from its start with twice the pool; the tallies are those of
                                  a run with a large enough pool */
} cm_run_stats;

/* back/fwd: [npix * hist_stride] counts, index = histogram bin + 1 (0 = underflow,
 * nbins + 1 = overflow), exactly Histogram::counts(bin) of the reference
 * (Utility/Histogram.cu:73-116).  All host pointers. */
int cm_run(cm_context* ctx, const cm_run_desc* desc, uint32_t* back, uint32_t* fwd, cm_run_stats* stats);
/* Same with inputs (pixel arrays) and outputs (back, fwd) already in device memory. */
int cm_run_device(cm_context* ctx, const cm_run_desc* desc_device_arrays, uint32_t* back_device, uint32_t* fwd_device,
                  cm_run_stats* stats, void* stream);

/* Autotuner: times the transport loop of desc (host arrays as for cm_run; its tallies are discarded)
 * under candidate settings, one setting at a time from the defaults (coordinate descent; a change is
 * kept when it is at least 1 % faster; passes repeat, at most 3, until one changes nothing), and keeps
 * the fastest for this context's later runs.  desc
 * should hold at least a wave's worth of primaries so that the trial sees the full and the tail phases
 * of a run.  The settings are kept for desc->precision; *best (may be NULL) receives them. */
int cm_autotune(cm_context* ctx, const cm_run_desc* desc, cm_tuning* best);

/* No counterpart in the reference.  cm_run_device for callers that cannot
 * allocate device memory while they run: a service whose device memory belongs
 * to another allocator (a caching pool, a reservation fixed at start-up), where
 * a cudaMalloc would fail or upset that allocator's accounting.  This call
 * allocates nothing: its scratch is one fixed 32 MiB device array that the
 * library holds on every GPU that loads it until the process exits.  Same
 * arguments, same tallies as cm_run_device (stream 0 = the legacy default
 * stream; stats->kernel_ms stays zero).  Limits: npix <= 65536; the wave is
 * capped by the scratch (about 17 k electrons in FP32, 12 k in FP64), so a run
 * whose secondaries overflow the fixed pool returns CM_EOVERFLOW instead of
 * growing it.  The scene must already be on the device for desc->precision
 * (uploading it allocates): after the last scene change, make one cm_run,
 * cm_run_device or cm_eval_* call with that precision first, else CM_ESTATE.
 * The first call on a device looks up the array's device address; make that
 * first call before any stream capture.  Every call, from any context on the
 * device, shares the one array and clears what must start at zero (counters,
 * tallies); calls whose work overlaps on the GPU race on it and must be
 * ordered by the caller. */
int cm_run_noalloc(cm_context* ctx, const cm_run_desc* desc_device_arrays, uint32_t* back_device,
                   uint32_t* fwd_device, cm_run_stats* stats, void* stream);

/* ---- job server: streams of scan jobs --------------------------------------
 * The reference runs one LinesOnLayers scan at a time on one thread
 * (JMONSELTests/LinesOnLayers.cu:327-398).  A server batches jobs continuously
 * on one GPU: the jobs of one precision and set of run options share one
 * resident wave of electrons, one merged scene (each job's chamber and regions
 * appended, or shared with an earlier job of the same geometry; tables,
 * materials and scatter models shared when equal) and one set
 * of pixel tables and tallies.  Queued jobs are admitted first in, first out
 * while fewer than `slots` jobs are in their batch and the job's pixel and
 * tally buffers fit in `budget_gb` beside the running jobs'; an admitted job's
 * primaries join the wave as soon as those of the jobs before it have started,
 * so jobs that arrive while others are on the GPU fill the room their ending
 * cascades leave.  A job is done when its primaries have started and its
 * electrons have all ended.  A job is a scene (copied from `scene` at
 * submission, which the caller may then reuse) and a run description with HOST
 * arrays (copied; energy histograms only).  Its tallies depend only on its
 * scene, pixels and stream keys: the same alone, in any mix and through cm_run. */
typedef struct cm_server cm_server;

#define CM_JOB_QUEUED 0
#define CM_JOB_RUNNING 1
#define CM_JOB_DONE 2
#define CM_JOB_FAILED 3
#define CM_JOB_CANCELLED 4

typedef struct {
  int state;                       /* CM_JOB_* */
  int error;                       /* status of a failed or cancelled job */
  double submit_s, start_s, end_s; /* seconds on the server's clock */
  int64_t primaries, steps;        /* of a finished job */
} cm_job_info;

int cm_server_create(int device, int slots, double budget_gb, cm_server** out);
/* launch settings (as cm_set_tuning) of the server's batches of one precision, taken by the batches that
 * start after the call */
int cm_server_tune(cm_server* server, int precision, const cm_tuning* tuning);
/* stops the batches after their current round of iterations and frees everything */
int cm_server_destroy(cm_server* server);
int cm_job_submit(cm_server* server, const cm_context* scene, const cm_run_desc* desc, int* out_job);
int cm_job_poll(cm_server* server, int job, cm_job_info* info);
/* waits until the job has ended or timeout_s passed (timeout_s < 0: no limit) */
int cm_job_wait(cm_server* server, int job, double timeout_s, cm_job_info* info);
/* a queued job is dropped; a running one starts no more primaries after the current round of iterations
 * and ends CANCELLED once its electrons in flight have ended */
int cm_job_cancel(cm_server* server, int job);
/* copies a finished job's tallies ([npix * hist_stride] each, may be NULL) and stats, then forgets the job;
 * a failed or cancelled job returns its error */
int cm_job_result(cm_server* server, int job, uint32_t* back, uint32_t* fwd, cm_run_stats* stats);

/* ---- per-function entry points (parity checks; host arrays, SI units) -------
 * Deviates are injected from u arrays so that each result can be compared
 * with the reference on the same inputs.  precision selects the kernel. */
/* NISTMottRS::totalCrossSection / randomScatteringAngle (JMONSEL/NISTMottRS.cu:103-154) of method 1..3; u[2n] */
int cm_eval_nistmott(cm_context* ctx, int Z, int method, int n, const double* E, const double* u, double* sigma, double* theta,
                     int precision);
/* NUTableInterpolation::interpolate (JMONSEL/NUTableInterpolation.cu:98-115); x[3n] */
int cm_eval_table(cm_context* ctx, int table, int n, const double* x, int order, double* out, int precision);
/* The windows that interpolation selects, NULagrangeInterpolation::locate per axis
 * (JMONSELutils/NULagrangeInterpolation.cu:5-68): out[6n] = (first index, nearest index) for axes 0..2,
 * -1 for axes the table does not have; x[3n] and order as for cm_eval_table (order applies to 1-D tables). */
int cm_eval_locate(cm_context* ctx, int table, int n, const double* x, int order, int* out, int precision);
/* MONSEL_MaterialScatterModel::scatter's choice of mechanism (MONSEL_MaterialScatterModel.cu:93-134):
 * in[2n] = E (J), deviate u; out[2n] = (index of the mechanism in the order it was added, or -1 when
 * the model has no rate; total scatter rate in 1/m) */
int cm_eval_pick(cm_context* ctx, int msm, int n, const double* in, double* out, int precision);
/* TabulatedInelasticSM::scatterRate + scatter (JMONSEL/TabulatedInelasticSM.cu:209-459);
 * in[9n] = E theta phi u0..u5, out[12n] = rate E' dx dy dz hasSE ESE sdx sdy sdz ndev 0 */
int cm_eval_tabulated(cm_context* ctx, int msm, int mech, int n, const double* in, double* out, int precision);
/* SelectableElasticSM::scatterRate + scatter (JMONSEL/SelectableElasticSM.cu:42-67);
 * in[7n] = E theta phi u0..u3, out[6n] = rate dx dy dz Z ndev */
int cm_eval_elastic(cm_context* ctx, int msm, int mech, int n, const double* in, double* out, int precision);
/* JoyLuoNieminenCSD::compute, FittedInelSM and polaron rates of a PMMA-like model;
 * in[2n] = E len, out[3n] */
int cm_eval_csd(cm_context* ctx, int msm, int n, const double* in, double* out, int precision);
/* GanachaudMokraniPhononInelasticSM (JMONSEL/GanachaudMokraniPhononInelasticSM.cu:19-72);
 * in[5n] = E theta phi u0 u1, out[6n] = rate E' dx dy dz Eprev */
int cm_eval_phonon(cm_context* ctx, int msm, int mech, int n, const double* in, double* out, int precision);
/* NormalShape::getFirstNormal, Shape::contains(p0) and NormalShape::contains(p0, p1) (double precision);
 * p01[6n], out[6n] = nx ny nz u contains(p0) contains(p0,p1) */
int cm_eval_shape(cm_context* ctx, int shape, int n, const double* p01, double* out);
/* ExpQMBarrierSM::barrierScatter + the nudge of MonteCarloSS::takeStep
 * (JMONSEL/ExpQMBarrierSM.cu:50-219); in[6n] = E theta phi x y z, out[7n] = E' dx dy dz x y z ... see implementation */
int cm_eval_barrier(cm_context* ctx, int from_region, int to_region, int n, const double* in, double* out, int precision);
/* MONSEL_MaterialScatterModel::randomMeanPathLength (MONSEL_MaterialScatterModel.cu:64-91); in[2n] = E u */
int cm_eval_freepath(cm_context* ctx, int msm, int n, const double* in, double* out, int precision);

#ifdef __cplusplus
}
#endif
#endif
