/* qvti.h -- C ABI of the B200 viscoelastic pseudospectral time stepper.
 *
 * Extended, status-returning entry points.  The reference exposes its path
 * only through the void functions of Myfunctions.h (cuda_Device_malloc,
 * cuda_Host_initialization, cuda_forward_acoustic_3D, cuda_Device_free);
 * those are provided unchanged in include/Myfunctions.h and are built on the
 * functions below.  Each declaration names the reference interface whose
 * role it takes (file:line within the reference project).
 *
 * Conventions (the reference's): fields are float32 [ix][iy][iz], z fastest,
 * on the total padded grid ntx*nty*ntz with `pml` C-PML cells on each face;
 * seismograms are [it][ir].  All functions return QVTI_OK (0) or an error
 * code; qvti_last_error() reports the last failure of the calling process.
 * Plain pointers and sizes only.
 */
#ifndef QVTI_H
#define QVTI_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    QVTI_OK = 0,
    QVTI_ERR_ARG = 1,         /* invalid argument                          */
    QVTI_ERR_CUDA = 2,        /* CUDA runtime error                        */
    QVTI_ERR_UNSUPPORTED = 3, /* grid size / option not supported          */
    QVTI_ERR_STATE = 4,       /* call out of order (e.g. no model set)     */
    QVTI_ERR_OOM = 5,         /* device allocation failed                  */
    QVTI_ERR_NONFINITE = 6,   /* a non-finite value was detected           */
    QVTI_ERR_TIMEOUT = 7      /* a wait ended before its shot finished     */
};

enum { QVTI_SRC_FORCE_X = 0, QVTI_SRC_EXPLOSIVE = 1 };

typedef struct qvti_sim qvti_sim;

typedef struct {
    int ntx, nty, ntz;  /* total padded grid (PML inside), each even, >= 16, 2/3/5/7-smooth */
    int pml;            /* C-PML thickness in cells on every face                           */
    float dx, dy, dz;   /* grid spacing (m)                                                 */
    float dt;           /* time step (s)                                                    */
    float f0;           /* reference / source frequency (Hz); w0 = 2 pi f0                   */
    int vti;            /* 0 isotropic, 1 VTI (Thomsen eps, delta; c66 = c44)               */
    int device;         /* CUDA device ordinal                                              */
    float w0;           /* constant-Q reference angular frequency; 0 = 2 pi f0 with the
                           reference's pi (viscoelas_3D.cpp:109)                              */
} qvti_config;

/* Device memory the engine needs for a grid with `pml` C-PML cells per face
 * (bytes; the C-PML memory variables are stored for their slabs only).
 * Replaces the sizing implicit in cuda_Device_malloc
 * (cuviscoelas_3D.cu:1689-1916). */
size_t qvti_footprint_bytes(int ntx, int nty, int ntz, int pml, int vti);

/* Allocate a simulation on cfg->device.  Replaces cuda_Device_malloc
 * (Myfunctions.h:91-96, cuviscoelas_3D.cu:1689-1916). */
int qvti_create(const qvti_config* cfg, qvti_sim** out);

/* Free everything.  Replaces cuda_Device_free (Myfunctions.h:98-102,
 * cuviscoelas_3D.cu:1922-2141). */
int qvti_destroy(qvti_sim* sim);

/* The configuration a simulation was created with.  Lets a caller reuse a
 * simulation for the next shot when grid, spacing, dt and frequency are
 * unchanged, as the reference reuses the buffers of cuda_Device_malloc across
 * its shot loop (viscoelas_3D.cpp:355-405). */
int qvti_get_config(const qvti_sim* sim, qvti_config* cfg);

/* Number of simulations qvti_create has made in this process (diagnostics:
 * shows whether a shot loop allocates per shot).  No counterpart in the
 * reference. */
long long qvti_sims_created(void);

/* Set the model: velp, vels, rho, gama_p = atan(1/Qp)/pi, gama_s (and eps,
 * delta when vti) as ntp floats each, host pointers (on_device = 0) or device
 * pointers (on_device = 1).  Builds the constant-Q, C-PML and k-space tables
 * in FP64 on the GPU.  Host arrays are staged in the simulation's own
 * scratch (no device allocation); the call returns once they have been
 * read.  Replaces the model H2D copies and the setup kernels of
 * cuda_forward_acoustic_3D (cuviscoelas_3D.cu:1179-1230). */
int qvti_set_model(qvti_sim* sim, const float* velp, const float* vels, const float* rho, const float* gama_p,
                   const float* gama_s, const float* eps, const float* delta, int on_device);

/* Source: type QVTI_SRC_FORCE_X adds wavelet[it] to vx at (s_ix, s_iy, s_iz)
 * after the stress update of step it (cuviscoelas_3D.cu:772-777);
 * QVTI_SRC_EXPLOSIVE adds it to pxx, pyy, pzz instead (the reference's
 * commented explosive variant, cu:775-776).  s_iz is the injection index
 * itself (the reference-compatible cuda_forward_acoustic_3D adds its +10).
 * wavelet: nt host floats; nt also sizes the seismogram buffers. */
int qvti_set_source(qvti_sim* sim, int type, int s_ix, int s_iy, int s_iz, const float* wavelet, int nt);

/* Receivers at depth index r_iz and padded positions (r_ix[i], r_iy[i]),
 * rn of them, host arrays (cuviscoelas_3D.cu:782-791). */
int qvti_set_receivers(qvti_sim* sim, int r_iz, const int* r_ix, const int* r_iy, int rn);

/* Zero the wavefield, memory variables and step counter
 * (cuda_kernel_initialization, cuviscoelas_3D.cu:312-410). */
int qvti_reset(qvti_sim* sim);

/* Advance nsteps time steps asynchronously (the body of the time loop,
 * cuviscoelas_3D.cu:1255-1630), replayed from a captured CUDA graph. */
int qvti_step(qvti_sim* sim, int nsteps);

/* Advance nsteps steps and report their device time in milliseconds,
 * measured with CUDA events on the simulation's stream (synchronous). */
int qvti_step_timed(qvti_sim* sim, int nsteps, float* ms);

/* Wait for all queued work. */
int qvti_sync(qvti_sim* sim);

/* Number of steps advanced since the last reset. */
int qvti_steps_done(const qvti_sim* sim);

/* Copy the seismograms recorded so far (steps_done x rn each, [it][ir]) to
 * host memory (cuviscoelas_3D.cu:1640-1645). Any pointer may be NULL. */
int qvti_get_records(qvti_sim* sim, float* vx, float* vy, float* vz);

/* Copy `count` wavefields starting at `first` in the order
 * vx vy vz pxx pyy pzz pxy pxz pyz to host memory (count*ntp floats);
 * snapshots (the reference's dead snapshot block, cu:1611-1627). */
int qvti_get_fields(qvti_sim* sim, int first, int count, float* out);

/* Device pointer of wavefield `which` (same order) for in-HBM consumers. */
int qvti_device_field(qvti_sim* sim, int which, float** dev_ptr);

/* Sum of squares of every wavefield (FP64 reduction on the device): the
 * per-run energy-norm check; also flags non-finite values. */
int qvti_field_norms(qvti_sim* sim, double* norms9, int* nonfinite);

/* Non-finite sentinel: queue, on the simulation's stream, a check of the
 * particle velocities (a NaN or Inf anywhere reaches them within a step:
 * every derivative is a global transform).  A hit sets a device flag that
 * stays set until qvti_reset; when host_flag is not NULL (pinned host memory)
 * the flag is copied there in stream order, so it is valid once work queued
 * after this call has completed.  Asynchronous; the scheduler runs it after
 * every chunk of steps and ends a shot with QVTI_ERR_NONFINITE.  The
 * reference checks nothing (cuviscoelas_3D.cu:1255-1630). */
int qvti_check_finite_async(qvti_sim* sim, int* host_flag);

/* Checkpoint / resume.  A snapshot holds everything a step reads that an
 * earlier step wrote: particle velocities, stresses, the z-derivative
 * accumulators carried into the next velocity update, the loss potentials
 * and the C-PML memory variables (55 full-grid arrays), the step count and
 * the seismograms recorded so far.  The model, source wavelet and receivers
 * are inputs, not state: set them on the resuming simulation as for the
 * original run (the reference declares checkpoint variables but never uses
 * them, viscoelas_3D.cpp:223-229).  Resuming is bitwise: steps run after
 * qvti_load_state give exactly the records and wavefields of an
 * uninterrupted run.
 *
 * qvti_state_bytes: size of a snapshot of this simulation at its current
 * step.  qvti_save_state: copies the snapshot into `host` (at least that
 * many bytes), after the simulation's queued steps.  qvti_load_state:
 * restores a snapshot; QVTI_ERR_ARG if the buffer is not a snapshot, or was
 * taken on another grid, spacing, dt, C-PML width or medium type, or holds
 * more recorded steps or another receiver count than this simulation's
 * source and receivers allow; QVTI_ERR_STATE before a source is set. */
int qvti_state_bytes(qvti_sim* sim, size_t* bytes);
int qvti_save_state(qvti_sim* sim, void* host, size_t bytes);
int qvti_load_state(qvti_sim* sim, const void* host, size_t bytes);

/* One whole shot with host buffers, synchronous: model upload, setup,
 * nt steps, seismogram download.  The reference-call semantics of
 * cuda_forward_acoustic_3D (Myfunctions.h:77-85, cuviscoelas_3D.cu:1137-1652)
 * with an explicit injection index. rec_* receive nt*rn floats each.
 * Inside the call the model upload and the state clear are queued without
 * waiting, so the step graphs are built on the host while the model moves;
 * the results equal qvti_set_model + qvti_set_receivers + qvti_set_source +
 * qvti_reset + qvti_step + qvti_get_records bit for bit. */
int qvti_forward_shot(qvti_sim* sim, const float* velp, const float* vels, const float* rho, const float* gama_p,
                      const float* gama_s, const float* eps, const float* delta, int src_type, int s_ix, int s_iy,
                      int s_iz, const float* wavelet, int nt, int r_iz, const int* r_ix, const int* r_iy, int rn,
                      float* rec_vx, float* rec_vy, float* rec_vz);

/* 1D staggered spectral derivative of a host field along `axis` (0 x, 1 y,
 * 2 z) with the forward (fwd=1, i k e^{+ik d/2}) or backward shift; the
 * building block of the velocity update (cuviscoelas_3D.cu:707-744 with the
 * transforms it feeds).  For tests and diagnostics. */
int qvti_derivative_1d(qvti_sim* sim, int axis, int fwd, const float* in, float* out);

/* One constant-Q derivative field of a host field: out = Re IFFT3(|k|^power
 * T(k_axis) FFT3(in)) / ntp, power in {-1, 0, 1} (the reference's Ap1, Ap2,
 * Ap3, cuviscoelas_3D.cu:188-190) and T the forward (fwd=1) or backward
 * staggered shift along `axis` -- one of the 45 fields of
 * cuviscoelas_3D.cu:1342-1562 on its own.  For tests and diagnostics. */
int qvti_q_derivative(qvti_sim* sim, int axis, int fwd, int power, const float* in, float* out);

/* qvti_q_derivative for callers that cannot allocate device memory: a
 * serving process with a footprint fixed at start-up, a host framework that
 * hands out pre-planned buffers from its own pool, or a latency-critical loop
 * that cannot absorb the device-wide synchronisation of cudaMalloc/cudaFree.
 * No counterpart in the reference.
 *   d_in, d_out: device arrays of ntx*nty*ntz floats (caller-owned); the
 *   result is written to d_out asynchronously on `stream` (a cudaStream_t,
 *   NULL for the default stream).
 * Nothing is allocated: the scratch half spectrum and the 1D tables live in
 * fixed-size device arrays of the library, held by every GPU that loads it
 * until the process exits.  Limits: each dimension even, 16..1024 and
 * 2/3/5/7-smooth, and (ntz/2 + 1)*ntx*nty <= 524288 (4 MiB of scratch, e.g.
 * 96^3 or 64x64x128); larger grids return QVTI_ERR_UNSUPPORTED.  The first
 * call on a device looks up the arrays' device addresses (and sets kernel
 * attributes) -- make it before any stream capture.  All calls on a device
 * share one scratch, which keeps the last call's contents (nothing in it
 * needs clearing): calls that can overlap on the GPU (different streams,
 * no ordering between them) race and must not be issued. */
int qvti_q_derivative_noalloc(const float* d_in, float* d_out, int ntx, int nty, int ntz, float dx, float dy,
                              float dz, int axis, int fwd, int power, void* stream);

/* Per-kernel device time of the time step: runs nrep steps (advancing the
 * state) with CUDA events between their kernels; sets *nkernels to the
 * kernels per step and fills names (maxk*32 chars), the average ms per launch
 * and each kernel's algorithmic HBM bytes per launch (maxk >= *nkernels).
 * No counterpart in the reference, whose only timing is the CPU clock()
 * around the whole program (viscoelas_3D.cpp:70-74, 472-480). */
int qvti_profile_step(qvti_sim* sim, int nrep, int maxk, int* nkernels, char* names, float* ms, double* bytes);

/* The simulation's CUDA stream (cudaStream_t), for callers that order their
 * own work after its steps.  The reference keeps one stream per device
 * inside struct MultiGPU (cuviscoelas_3D.cu:1168). */
int qvti_get_stream(qvti_sim* sim, void** stream);

/* kz planes per batch of the k-space passes (1..nz/2+1); a tuning knob for
 * qvti_autotune.  No counterpart in the reference. */
int qvti_set_kz_batch(qvti_sim* sim, int kz_batch);

/* Form of the transforms.  QVTI_FORM_PLAIN: every FFT stage as FP32
 * butterflies.  QVTI_FORM_TC: the 256-point y transforms (forward and
 * inverse, the reference's cufftExecC2C work of cuviscoelas_3D.cu:1272-1562
 * along y) as split-precision tensor-core contractions -- each radix-16
 * stage a 16-point DFT matrix product on tcgen05 with TF32 hi/lo operands
 * (three products, FP32 accumulation); the other transforms stay FP32.
 * QVTI_ERR_UNSUPPORTED when the grid's y length is not 256.  A device-side
 * wait that times out makes the next qvti_sync / qvti_get_records return
 * QVTI_ERR_TIMEOUT.  No counterpart in the reference. */
enum { QVTI_FORM_PLAIN = 0, QVTI_FORM_TC = 1 };
int qvti_set_form(qvti_sim* sim, int form);

/* Tile of each step kernel, in the order QVTI_TILE_*: the z rows of a k_vy
 * or k_vx block, the y rows of a k_fz, k_mx or k_sigma block, the lines of
 * a k_cy block.  tiles[i] = 0 keeps kernel i's default (its compiled
 * kernel's tile where the transform length has one); tiles[i] > 0 runs the
 * runtime-length kernel with that tile: even, 2..32, dividing the axis it
 * tiles (k_cy: any), and the step's shared memory within the device limit,
 * else QVTI_ERR_UNSUPPORTED and the tiling is unchanged.  The results agree
 * with the default tiling to FP32 rounding.  A tuning knob of
 * qvti_autotune_tiles; no counterpart in the reference. */
enum { QVTI_TILE_VY = 0, QVTI_TILE_VX, QVTI_TILE_FZ, QVTI_TILE_CY, QVTI_TILE_MX, QVTI_TILE_SIGMA, QVTI_NUM_TILES };
int qvti_set_tiles(qvti_sim* sim, const int tiles[QVTI_NUM_TILES]);
/* The tiles the step launches take and, per kernel, 1 where it runs its
 * runtime-length kernel (either may be null). */
int qvti_get_tiles(qvti_sim* sim, int tiles[QVTI_NUM_TILES], int runtime[QVTI_NUM_TILES]);

/* Per-kernel tile search on a simulation whose model and source are set:
 * for each step kernel, its default and the runtime-length kernel at every
 * valid tile in {2, 4, 8, 16, 32}, each timed over probe_steps profiled
 * steps (CUDA events between the kernels) after a reset and one warm-up
 * step, the kernels already searched at their chosen tiles, the rest at
 * their defaults; a tile other than the default is taken only when it is at
 * least 3 % faster.  Leaves the chosen tiling set and the simulation reset.
 * best[i]: the chosen setting (0 = default), ms[i]: its time (either may be
 * null).  Needs nt >= probe_steps + 1 steps of wavelet capacity.  No
 * counterpart in the reference. */
int qvti_autotune_tiles(qvti_sim* sim, int probe_steps, int best[QVTI_NUM_TILES], float ms[QVTI_NUM_TILES]);

/* Failure-path check of the device-side bounded waits: queue on the
 * simulation's stream a wait (0 < seconds <= 2) on a barrier nothing
 * completes; when it runs out it records QVTI_ERR_TIMEOUT in the same device
 * flag a stalled tensor-core round would, so the next qvti_sync returns
 * QVTI_ERR_TIMEOUT; qvti_reset clears it and the simulation stays usable.
 * No counterpart in the reference. */
int qvti_probe_bounded_wait(qvti_sim* sim, double seconds);

/* ---------------------------------------------------------------------
 * Reverse-time migration and Q compensation.  The reference declares these
 * as flags only (viscoelas_3D.cpp:1-3 "viscoacoustic reverse time
 * migration", :42-65 RTM_type, imaging_condition, media_type, :223-229
 * checkpoints) and implements none of them.
 * --------------------------------------------------------------------- */
enum {
    QVTI_MEDIA_VISCOELASTIC = 1,   /* dispersion and loss (the default)                    */
    QVTI_MEDIA_DISPERSION_ONLY = 2, /* constant-Q dispersion, loss terms off                */
    QVTI_MEDIA_LOSSLESS = 3,        /* gamma = 0: elastic (built by qvti_set_model)         */
    QVTI_MEDIA_Q_COMPENSATED = 4    /* loss terms with reversed sign: amplitude compensation
                                       for back-propagation (unstable over long distances at
                                       high frequency, as any amplitude-amplifying operator) */
};
/* Medium of the stepping (viscoelas_3D.cpp:59-63's media_type).  Call before
 * qvti_set_model (the lossless medium changes the coefficients it builds). */
int qvti_set_media(qvti_sim* sim, int media);

/* Back-propagation source: from the next step on, step it adds sample
 * nt - 1 - it of each given component (host arrays of nt x rn floats,
 * [it][ir] like the records; any may be NULL) to that velocity component at
 * receiver ir, where the records are taken (the adjoint of recording).  Set
 * after qvti_set_receivers; nt = 0 clears it. */
int qvti_set_injection(qvti_sim* sim, const float* vx, const float* vy, const float* vz, int nt);

typedef struct {
    int media;        /* QVTI_MEDIA_* of both propagations                          */
    int snap_every;   /* imaging interval: correlate every snap_every-th step      */
    float illum_eps;  /* source-normalised image: I / (illumination + eps max illum) */
} qvti_rtm_opts;

/* One shot of reverse-time migration: the source wavefield is propagated
 * forward and its velocities kept on the device every opts->snap_every steps;
 * the observed records (nt x rn per component; NULL components are not
 * injected) are propagated backward in time from the receivers; at the kept
 * steps the zero-lag cross-correlation image sum_t sum_c S_c R_c
 * (imaging_condition 4) and the source illumination sum_t sum_c S_c^2 are
 * accumulated on the device.  image_xcorr and image_norm (the cross-
 * correlation divided by the illumination plus opts->illum_eps times its
 * maximum, imaging_condition 3) receive ntx*nty*ntz floats each (either may
 * be NULL).  QVTI_ERR_OOM if the kept source velocities do not fit;
 * QVTI_ERR_NONFINITE if a propagation blew up (the Q-compensated medium
 * over long paths through strong attenuation). */
int qvti_rtm_shot(const qvti_config* cfg, const float* velp, const float* vels, const float* rho, const float* gama_p,
                  const float* gama_s, const float* eps, const float* delta, int src_type, int s_ix, int s_iy, int s_iz,
                  const float* wavelet, int nt, int r_iz, const int* r_ix, const int* r_iy, int rn,
                  const float* obs_vx, const float* obs_vy, const float* obs_vz, const qvti_rtm_opts* opts,
                  float* image_xcorr, float* image_norm);

/* ---------------------------------------------------------------------
 * Batches and serving.  The reference runs shots one after another from a
 * host loop (viscoelas_3D.cpp:355-405, one cuda_forward_acoustic_3D call per
 * shot, cuviscoelas_3D.cu:1163-1629); these entry points run many shots of
 * uneven size on one GPU at once, each on its own stream with its time loop
 * as CUDA-graph launches, admitted first-in first-out under an HBM budget.
 * Shots are independent, so each shot's result is the same whether it runs
 * alone or among others.
 * --------------------------------------------------------------------- */
typedef struct {
    int ntx, nty, ntz, pml;       /* as qvti_config                                   */
    float dx, dy, dz, dt, f0;
    int vti;
    const float *velp, *vels, *rho, *gama_p, *gama_s; /* host, ntx*nty*ntz each      */
    const float *eps, *delta;     /* host, VTI only (NULL otherwise)                  */
    int src_type, s_ix, s_iy, s_iz; /* as qvti_set_source                             */
    const float* wavelet;         /* nt samples                                       */
    int nt;                       /* steps                                            */
    int r_iz, rn;                 /* as qvti_set_receivers                            */
    const int *r_ix, *r_iy;
    float *rec_vx, *rec_vy, *rec_vz; /* host outputs, nt*rn floats each, [it][ir]; may be NULL */
} qvti_shot;

typedef struct {
    int status;        /* QVTI_OK or this shot's error                          */
    double queue_s;    /* submit -> its steps enqueued on the GPU (host clock)  */
    double latency_s;  /* submit -> records copied out (host clock)             */
    float device_ms;   /* first to last step of the shot on the GPU (CUDA events) */
} qvti_shot_result;

/* Admission order of waiting shots.  QVTI_SCHED_FIFO: first submitted,
 * first admitted.  QVTI_SCHED_SMALLEST_FIRST: the waiting shot with the
 * fewest cell-steps (ntx nty ntz nt; ties by submission) is admitted next,
 * which shortens the typical latency of a mix of small and large shots;
 * the oldest waiting shot is admitted next once smaller ones have passed it
 * 8 times, so large shots are delayed, not starved. */
enum { QVTI_SCHED_FIFO = 0, QVTI_SCHED_SMALLEST_FIRST = 1 };

typedef struct {
    int device;        /* CUDA device ordinal                                   */
    size_t mem_budget; /* device bytes the scheduler may hold; 0: 90% of free   */
    int max_active;    /* shots in flight; 0: per grid from qvti_autotune        */
    int policy;        /* QVTI_SCHED_FIFO or QVTI_SCHED_SMALLEST_FIRST           */
} qvti_sched_opts;

typedef struct qvti_server qvti_server;

/* Start a serving loop (one scheduler thread) on opts->device. */
int qvti_server_create(const qvti_sched_opts* opts, qvti_server** out);

/* Queue one shot.  Every array the descriptor points to is borrowed until
 * qvti_server_wait has returned its ticket.  A shot whose footprint exceeds
 * the whole budget is rejected with QVTI_ERR_OOM. */
int qvti_server_submit(qvti_server* srv, const qvti_shot* shot, long long* ticket);

/* Wait for a ticket (timeout_s < 0: no limit).  QVTI_ERR_TIMEOUT if the shot
 * has not finished in time (the ticket stays valid); otherwise the shot's
 * result (res->status carries its own error). */
int qvti_server_wait(qvti_server* srv, long long ticket, double timeout_s, qvti_shot_result* res);

/* Shots waiting plus in flight, and the device bytes the pool holds. */
int qvti_server_load(qvti_server* srv, int* queued, int* active, size_t* pool_bytes);

/* Finish the shots already submitted, stop the loop, free the pool. */
int qvti_server_destroy(qvti_server* srv);

/* Run n shots through a serving loop and wait for all; results[n] and the
 * wall time of the whole batch (host clock). */
int qvti_run_batch(const qvti_shot* shots, int n, const qvti_sched_opts* opts, qvti_shot_result* results,
                   double* wall_s);

/* Probe one grid: the form of the transforms (plain FP32 stages, or the
 * tensor-core DFT plan where the grid has one) with one shot in flight, the
 * per-kernel tiles in that form (qvti_autotune_tiles), then probe_steps
 * steps on 1..max_active concurrent simulations (homogeneous model) for
 * each kz batch in {nz/2+1, (nz/2+2)/2}; report the fastest setting and its
 * Gcell-steps/s.  The scheduler caches the result per grid and applies it
 * to the shots of that grid.  No counterpart in the reference, which runs
 * one shot at a time (viscoelas_3D.cpp:355-405). */
typedef struct {
    int active;          /* shots in flight                                   */
    int kz_batch;        /* kz planes per batch of the k-space passes         */
    int form;            /* QVTI_FORM_PLAIN or QVTI_FORM_TC                   */
    double gcell_steps;  /* measured Gcell-steps/s of that setting            */
    int tiles[QVTI_NUM_TILES]; /* per-kernel tiles (qvti_set_tiles)           */
} qvti_tuning;
int qvti_autotune_ex(const qvti_config* cfg, int max_active, int probe_steps, qvti_tuning* best);

/* qvti_autotune_ex without the form in the result. */
int qvti_autotune(const qvti_config* cfg, int max_active, int probe_steps, int* best_active, int* best_kz_batch,
                  double* gcell_steps);

/* Last error code of the calling thread and its description. */
int qvti_last_error(void);
const char* qvti_error_string(int code);

#ifdef __cplusplus
}
#endif
#endif
