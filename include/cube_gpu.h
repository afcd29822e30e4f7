/*
 * cube_gpu.h -- C ABI of the B200 P3M gravity step of CUBE: one image (nn=1), or
 * the box split into z-slabs over ranks (cube_params.nslab).
 *
 * The reference drives its step with zero-argument Fortran subroutines that share
 * module globals (main.f90:33-38: timestep, drift, buffer_grid, buffer_x, kick,
 * buffer_v).  This header replaces that sequence with explicit calls on an opaque
 * context.  Every entry point returns 0 on success or a negative CUBE_E_* code;
 * cube_gpu_last_error() gives the text.  A Fortran host binds these through an
 * ISO_C_BINDING interface module (see the integration notes); a Python host binds
 * them with ctypes (cube_nu_b200/_lib.py).
 *
 * Conventions
 *  - Arrays cross the boundary in the reference's own memory layout: xp(3,np) and
 *    vp(3,np) are Fortran column-major, i.e. three consecutive values per particle;
 *    rhoc(nt,nt,nt,nnt,nnt,nnt) is the physical coarse-cell count array of the
 *    checkpoint file `np` (checkpoint.f90:30), x fastest.
 *  - Particles are ordered as the reference stores them: tile (z,y,x outer), then
 *    coarse cell in the tile (x fastest), then arrival order (drift.f90:96-136).
 *  - Between cube_gpu_upload and cube_gpu_download the device owns the particle
 *    state; host buffers are only borrowed during those calls.
 *  - One host thread per context; never call from inside an OpenMP region.
 */
#ifndef CUBE_GPU_H
#define CUBE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Error codes (negative). */
#define CUBE_OK 0
#define CUBE_E_ARG (-1)        /* bad argument / inconsistent geometry                     */
#define CUBE_E_CUDA (-2)       /* CUDA runtime error                                       */
#define CUBE_E_CAPACITY (-3)   /* particle capacity or per-cell segment limit exceeded     */
#define CUBE_E_RANGE (-4)      /* particle moved beyond the ghost depth (drift.f90:64-73)  */
#define CUBE_E_COUNT (-5)      /* particle count not conserved (drift.f90:139-143)         */
#define CUBE_E_STATE (-6)      /* call out of order (e.g. step before upload)              */
#define CUBE_E_TIMEOUT (-7)    /* a bounded device-side wait gave up                       */
#define CUBE_E_COMM (-8)       /* a cube_comm callback failed (nslab > 1)                   */

/* Device error-word bits (set by kernels, read back by the host after a step). */
#define CUBE_DEVERR_DRIFT_RANGE 0x1u
#define CUBE_DEVERR_DEPOSIT_RANGE 0x2u
#define CUBE_DEVERR_INTERP_RANGE 0x4u
#define CUBE_DEVERR_SEGMENT 0x8u
#define CUBE_DEVERR_CAPACITY 0x10u
#define CUBE_DEVERR_FIXED_OVERFLOW 0x20u

/* Deposit arithmetic. */
#define CUBE_DEPOSIT_FP32 0  /* plain form: FP32 atomics (order-dependent rounding)           */
#define CUBE_DEPOSIT_FIXED 1 /* chosen form: int64 fixed-point atomics (deterministic)         */

/*
 * Run parameters.  Names and meanings follow parameters.f90; derived sizes
 * (nc, nt, ntt, ngp, ngt, nfp, nfb, nft; parameters.f90:57-69) are computed by the
 * library from these.  cube_params_default() fills the reference defaults.
 */
typedef struct cube_params {
  int64_t ng;        /* fine cells per dimension of the image (parameters.f90:24)       */
  int64_t ratio_cs;  /* fine cells per coarse cell, 4 (parameters.f90:25)               */
  int64_t nnt;       /* tiles per image per dimension (parameters.f90:28)               */
  int64_t nns;       /* subtiles per tile per dimension (parameters.f90:29)             */
  int64_t np_nc;     /* particles per coarse cell per dimension at the IC (:32)         */
  int64_t ncb;       /* coarse ghost depth, 4 (parameters.f90:81)                       */
  int64_t ngb;       /* PM2 tile buffer in fine cells, 16 (parameters.f90:61)           */
  int32_t izipx;     /* bytes per compressed coordinate: 1 (int8) or 2 (int16)          */
  int32_t pm3_on;    /* PM3 switch (kick.f90:9)                                         */
  int32_t pp_on;     /* PP switch (kick.f90:10)                                         */
  int32_t deposit_mode; /* CUBE_DEPOSIT_FP32 or CUBE_DEPOSIT_FIXED                     */
  float box;         /* box size in Mpc/h (parameters.f90:23)                           */
  float app;         /* PP softening in fine cells, 0.06 (parameters.f90:46)            */
  float apm1c;       /* PM1 softening in coarse cells, 3.5 (parameters.f90:38)          */
  float apm2;        /* PM2 softening in fine cells, 3.5 (parameters.f90:40)            */
  float apm3f;       /* PM3 softening in refined cells, 3.5 (parameters.f90:42)         */
  float mass_p_cdm;  /* particle mass in fine-cell units (ic.f90:839)                   */
  float f_nu;        /* neutrino mass fraction for the linear-response rescale (0: CDM) */
  int64_t np_capacity; /* particle capacity on device (0: derive from ng, np_nc)        */
  int32_t max_segment; /* largest destination cell the drift sorts in shared memory (0 or
                          above 16384: 16384); longer cells take a rank sort in HBM       */
  int32_t step_graph;  /* 1: cube_gpu_step replays each step as one captured CUDA graph   */
  int32_t pp_queue;    /* 1: PP as an autotuned work queue over cells (needs int8 codes, or
                          int16 with nt < 127); 0: one thread per particle                 */
  int32_t nslab;       /* z-slabs the periodic box is split into, one rank each (0 or 1: one
                          rank holds the whole box); nnt must be a multiple of nslab      */
  int32_t slab;        /* this rank's slab: tile layers [slab*L, (slab+1)*L) along z with
                          L = nnt/nslab; every other coarse cell is another rank's        */
  int32_t reserved[3];
} cube_params;

/* Per-step scalars chosen by the host timestep (timestep.f90:4-110). */
typedef struct cube_step_in {
  float dt;      /* kick step (timestep.f90:267)                  */
  float dt_old;  /* previous dt; drift uses (dt_old+dt)/2 (drift.f90:21) */
  float a_mid;   /* a at mid step (timestep.f90:297)              */
  float vz_max;  /* sim%vz_max from the previous kick (drift.f90:26)  */
} cube_step_in;

/* Per-step results that the reference writes into sim and tcat. */
typedef struct cube_step_out {
  float dt_pm1, dt_pm2, dt_pm3, dt_pp, dt_vmax; /* kick.f90:39,69,239,298,314 */
  float vmax[3];                                /* final |v| maxima              */
  float vz_max;                                 /* kick.f90:315                   */
  float f2max_pm1, f2max_pm2, f2max_pm3, f2max_pp;
  int32_t napm[8];                              /* PM3 class histogram, index 2..5 (kick.f90:132) */
  int64_t nplocal;
  int64_t pp_pairs;                             /* in-range PP pairs evaluated (both orders)  */
  float tcat[16];                               /* stage ms: 0 drift,1 PM1,2 PM2,3 PM3,4 PP,5 sum, 6 step wall on device */
  /* FP64 global reductions.  mass_pm*: the deposited density summed over the physical
   * cells of each level, in particle units (particle_mesh.f90:106 testrho, kick.f90:687-688
   * ptotal; the reference prints them at kick.f90:42,72,242): nplocal up to the rounding
   * of the TSC weights.  Exact int64 sums with CUBE_DEPOSIT_FIXED, FP64 sums of the FP32
   * weights otherwise.  mass_pm3 is 0 with PM3 off.  momentum: sum of vp over the
   * particles after the kick, per component, in FP64 (deterministic order). */
  double mass_pm1, mass_pm2, mass_pm3;
  double momentum[3];
  int64_t pp_candidates;                        /* PP candidate pairs tested (r^2 evaluated) */
} cube_step_out;

typedef struct cube_ctx cube_ctx;

/* Fill the reference defaults of parameters.f90 for a given ng. */
void cube_params_default(cube_params* p, int64_t ng);

/* Create a context on CUDA device `device`: derives sizes, builds the FP64 Green
 * tables on the device (Green/Green.f90:1-80, initialize.f90:247-334) and allocates
 * particle and mesh buffers.  Replaces initialize + create_cubefft_plan. */
int cube_gpu_create(const cube_params* p, int device, cube_ctx** out);
int cube_gpu_destroy(cube_ctx* ctx);

/* Copy particles in (particle_initialization.f90:77-90 after the checkpoint read). */
int cube_gpu_upload(cube_ctx* ctx, const void* xp, const float* vp, const int64_t* pid,
                    const int32_t* rhoc, int64_t nplocal);
/* Copy particles out (checkpoint.f90:24-33). `nplocal` receives the count. */
int cube_gpu_download(cube_ctx* ctx, void* xp, float* vp, int64_t* pid, int32_t* rhoc,
                      int64_t* nplocal);
/* Particles the context holds for its rank (sim%nplocal), the count a download returns;
 * negative on error. */
int64_t cube_gpu_nplocal(cube_ctx* ctx);

/* Zel'dovich initial conditions generated on the device (utilities/ic.f90), left as the
 * context's particle state (replaces reading the IC checkpoint).  The noise comes from
 * Philox4x32-10 keyed by `seed` (counter = Box-Muller pair index on the nic*ng grid);
 * pk_k/pk_p tabulate the linear P(k) at the IC redshift (k in h/Mpc, P in (Mpc/h)^3),
 * interpolated in log-log as ic.f90's interp_tf. */
typedef struct cube_ic_in {
  int32_t nic;       /* IC grid refinement (parameters.f90:33)            */
  int32_t npk;       /* table length                                       */
  uint64_t seed;
  float vfactor;     /* a^2 H(a) in code units (ic.f90:937-945)           */
  float reserved;
  const double* pk_k;
  const double* pk_p;
} cube_ic_in;
typedef struct cube_ic_out {
  int64_t nplocal;
  float grad_max[3]; /* max |gradphi| per axis on the lattice             */
  float vmax[3];     /* grad_max/(8 nic pi)*vfactor (ic.f90:584)           */
  float vz_max;
  float dt_vmax;     /* 0.9*16/max(vmax) (ic.f90:585)                     */
  int32_t nlayer;
  float mass_p_cdm;
} cube_ic_out;
int cube_gpu_ic(cube_ctx* ctx, const cube_ic_in* in, cube_ic_out* out);

/* ZIPV int16 velocity codec (utilities/pp_subtile.f90:61 decode, :125 encode; izipv=2,
 * vrel_boost=2.5): code = nint(65535*atan(sqrt(pi/2)/(sigma_vi*2.5)*v)/pi) and back.
 * Host arrays of n values, converted on the context's device. */
int cube_gpu_zipv_encode(cube_ctx* ctx, const float* v, int16_t* code, int64_t n, float sigma_vi);
int cube_gpu_zipv_decode(cube_ctx* ctx, const int16_t* code, float* v, int64_t n, float sigma_vi);
/* cube_gpu_download with the velocities written in the ZIPV int16 format (vp_code(3,np)). */
int cube_gpu_download_zipv(cube_ctx* ctx, void* xp, int16_t* vp_code, int64_t* pid, int32_t* rhoc,
                           int64_t* nplocal, float sigma_vi);

/*
 * Power spectrum of the device-resident particles, replacing the cicpower utility
 * (utilities/cicpower.f90:76-219) run on a checkpoint: CIC density on an nw^3 mesh,
 * delta = rho/mean - 1, then auto_power (utilities/powerspectrum.f90:140-210) with
 * up to n_corr pk_correction passes (powerspectrum.f90:212-259).  xi receives
 * xi(10,0:nbin) in the reference's layout (10 values per bin, bin 0 first):
 * 1 mode count, 2 mean k [h/Mpc], 3 raw power, 4 power minus shot noise, 5 aliasing-
 * corrected power [(Mpc/h)^3], 6-10 zero.  delta (NULL to skip) receives delta_c
 * (nw^3 floats, x fastest) as cicpower writes it.  With CUBE_DEPOSIT_FIXED the density
 * is summed in int64 fixed point (order independent).
 */
typedef struct cube_power_in {
  int32_t nw;       /* mesh side, ng*nic in cicpower (parameters.f90:73 with FFTFINE);
                       one of 16 32 48 64 96 128 144 192 256 288 432 512 576 1024      */
  int32_t n_interp; /* shot-noise window: 1 NGP, 2 CIC (as cicpower.f90:220 calls it), 3 TSC */
  int32_t n_int;    /* alias images per side in pk_correction, 3 in the reference (0..4) */
  int32_t n_corr;   /* pk_correction passes, 4 in the reference (powerspectrum.f90:198-201) */
} cube_power_in;

typedef struct cube_power_out {
  int64_t nbin;        /* nint(nyquist*sqrt(3)) (powerspectrum.f90:15)          */
  double mean;         /* particles per mesh cell, rho8/nw^3 (cicpower.f90:171) */
  float alpha;         /* slope of the last pk_correction pass (NaN: none ran)  */
  int32_t n_corr_done; /* pk_correction passes applied                          */
  float delta_min, delta_max;
  float ms;            /* device time of the call                               */
} cube_power_out;

int cube_gpu_power(cube_ctx* ctx, const cube_power_in* in, float* xi, int64_t nxi, float* delta,
                   cube_power_out* out);

/* drift.f90:1-233 with dt_mid=(dt_old+dt)/2; bit-exact arrival order and ZIPX update. */
int cube_gpu_drift(cube_ctx* ctx, const cube_step_in* in);
/* kick.f90:1-353: PM1 + PM2 + PM3 + PP velocity updates and dt criteria. */
int cube_gpu_kick(cube_ctx* ctx, const cube_step_in* in, cube_step_out* out);
/* One loop body of main.f90:36-38 (drift, ghosts, kick, ghosts). */
int cube_gpu_step(cube_ctx* ctx, const cube_step_in* in, cube_step_out* out);
/* The same step for a caller whose particle state lives in host memory, as the
 * reference's arrays xp, vp, PID, rhoc do between iterations of main.f90:30-59: uploads
 * the state from the four arrays (`nplocal` particles, checked as in cube_gpu_upload),
 * steps, and writes the new state back into the same arrays.  Equal to cube_gpu_upload +
 * cube_gpu_step + cube_gpu_download on those arrays; the copies the step does not wait
 * for overlap it (the ids go up and are reordered while the drift runs; positions, ids
 * and counts come down during the kick), which needs page-locked arrays.  After a failed
 * call the context holds no particles. */
int cube_gpu_step_host(cube_ctx* ctx, const cube_step_in* in, cube_step_out* out, void* xp, float* vp,
                       int64_t* pid, int32_t* rhoc, int64_t nplocal);

/* Inspection for tests.  cube_gpu_capture arms a capture: during the next kick the
 * field `what` (0: density = deposited mass per cell, 1: potential phi after the
 * inverse FFT and normalisation) of PM level `level` (1: the nc^3 mesh, 2: PM2 tile
 * `box`, 3: PM3 subtile `box` in initialize.f90:351-367 numbering) is copied aside.
 * cube_gpu_captured downloads it (x fastest, array index = reference index - m1)
 * and returns the number of values. */
int cube_gpu_capture(cube_ctx* ctx, int level, int box, int what);
int cube_gpu_captured(cube_ctx* ctx, float* out, int64_t n);
/* Opt-in per-kernel timers: CUDA events around every kernel launch on the context's
 * stream.  cube_gpu_profile(ctx, 1) resets and enables them; cube_gpu_profile_read
 * fills accumulated milliseconds and launch counts per kernel class (names from
 * cube_gpu_profile_name) and returns the number of classes. */
int cube_gpu_profile(cube_ctx* ctx, int enable);
int cube_gpu_profile_read(cube_ctx* ctx, double* ms, int64_t* count, int n);
const char* cube_gpu_profile_name(int i);
/* Queue PP shapes (cube_params.pp_queue).  The PP work is split by the occupancy of each
 * particle's coarse cell: cells of at most T particles take one thread per particle, the
 * others are cut into items of B particles that a persistent kernel pulls from a device
 * queue (largest cells first), staging candidates in shared-memory chunks of J.  The
 * library's autotuner times a sweep of shapes on the live state the first time a step
 * falls in occupancy class cls (largest cell <= 64, <= 512, <= 4096, larger: 0..3; the
 * reference's only tuning data is its PP timing, kick.f90:141-201) and keeps the fastest.
 * Forces do not depend on the shape.  cube_gpu_pp_shape sets the shape of a class (T <= 0
 * forgets it, so it is tuned again; B in {32, 64, 128, 256, 512}, J in 32..4096);
 * cube_gpu_pp_shape_get returns 1 and the shape and its timed milliseconds when the class
 * has one, else 0. */
int cube_gpu_pp_shape(cube_ctx* ctx, int cls, int T, int B, int J);
int cube_gpu_pp_shape_get(cube_ctx* ctx, int cls, int* T, int* B, int* J, double* ms);
/* Number of kernels this context has launched since creation. */
int64_t cube_gpu_kernel_launches(cube_ctx* ctx);

/* Real positions of the resident particles, replacing the int2real utility
 * (utilities/int2real.f90:68-86): xv(3,np) real(4) in coarse-cell units (0..nc),
 * the ZIPX offset plus the cell index, in the resident particle order. */
int cube_gpu_int2real(cube_ctx* ctx, float* xv, int64_t n);
/* Download the Green table of a level (1, 2, or 3 with class iapm 2..5). */
int cube_gpu_green_table(cube_ctx* ctx, int level, int iapm, float* out, int64_t n);
/* Asynchronous checkpoint (checkpoint.f90:11-39): the particle state as the context
 * stream leaves it (after the work issued so far) is copied to pinned staging memory on
 * a side stream, and a writer thread stores the five files of one image -- `info` gets
 * the caller's sim_header bytes (224 in the reference), `xp` int(izipx)(3,np), `vp`
 * real(4)(3,np), `np` int(4) rhoc, `id` int(8) PID -- while the host goes on stepping.
 * Steps that would overwrite the copied buffers wait for the copies on the device; the
 * host never waits.  One checkpoint is in flight at a time (a second call waits for the
 * first); cube_gpu_checkpoint_wait joins the writer and returns its status. */
typedef struct cube_ckpt_files {
  const char* info;
  const char* xp;
  const char* vp;
  const char* np;
  const char* id;
} cube_ckpt_files;
int cube_gpu_checkpoint_async(cube_ctx* ctx, const cube_ckpt_files* files, const void* header,
                              int64_t header_bytes);
int cube_gpu_checkpoint_wait(cube_ctx* ctx);

/* Neutrino linear response of the force kernels (kick.f90:23-29, get_tf_cb2matter).  The
 * host computes the per-step transfer ratio tf_F(k) on its k table as the reference does
 * (neutrinos/power_nu.f90:346-420) and passes log k (h/Mpc) and log tf_F, nb >= 3 points,
 * k increasing; every level's force kernel becomes interp_tf_F(|k|) * Gk (power_nu.f90:
 * 179-219, 449-498), rebuilt on the device before the next kick.  nb = 0 drops the table.
 * Without a table and with cube_params.f_nu > 0 the kernels are (1 - f_nu) * Gk
 * (initialize.f90:316-322), and PP uses (1 - f_nu)^2 (kick.f90:569).
 * cube_gpu_kernel_table downloads the kernel a level uses (as cube_gpu_green_table). */
int cube_gpu_nu_transfer(cube_ctx* ctx, const float* kh_log, const float* tf_log, int nb);
int cube_gpu_kernel_table(cube_ctx* ctx, int level, int iapm, float* out, int64_t n);
/* Download per-subtile PM3 class (ires, kick.f90:108-133), ns3 entries. */
int cube_gpu_subtile_class(cube_ctx* ctx, int32_t* ires, int64_t n);

/*
 * PM1 coarse density without allocating device memory.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc, such as a host whose
 * device memory is already held by another framework's caching pool (cudaMalloc would
 * fail or carve up memory the pool owns), or a caller on a latency-bound path where
 * cudaMalloc/cudaFree would synchronise the whole device.  It needs no context.
 *
 * xp (3 codes per particle, izipx bytes each), rhoc (nc^3 counts in the layout of
 * cube_gpu_upload) and rho (nc^3 floats, x fastest, global coarse cells) are device
 * pointers on the current device; the result is the PM1 density in mass units, the
 * same field cube_gpu_capture(ctx, 1, 0, 0) records during a kick (bit-identical
 * with CUBE_DEPOSIT_FIXED).  Work goes on `stream` (a cudaStream_t, NULL for the
 * default stream) and the call returns once that stream has finished it.
 *
 * All scratch lives in one static device array sized for at most
 * CUBE_NOALLOC_MAX_CELLS coarse cells and CUBE_NOALLOC_MAX_PARTICLES particles (about
 * 12 MB, held by every device that loads the library until the process exits); larger
 * sizes return CUBE_E_CAPACITY.  The 12 MB are committed when the library's device code
 * is first loaded on a device (with lazy module loading, at the first call of any entry
 * point there); a caller whose device memory a pool will later claim should make one
 * call on each device before the pool grows.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for the life of the
 * process: do not use the library on a device after cudaDeviceReset.  The call waits for
 * `stream` (it reads back a count), so it can never be recorded into a CUDA graph.  Every
 * call shares the array: calls that overlap on the GPU (other streams, other host
 * threads) race; serialise them.  Each call clears what it accumulates into.  Returns
 * CUBE_E_COUNT when rhoc holds a negative count or does not sum to np; on any error the
 * contents of rho are undefined.
 */
#define CUBE_NOALLOC_MAX_CELLS 262144       /* 64^3 coarse cells */
#define CUBE_NOALLOC_MAX_PARTICLES 2097152  /* 2^21 particles    */
int cube_gpu_pm1_density_noalloc(const cube_params* p, const void* xp, const int32_t* rhoc, int64_t np,
                                 float* rho, void* stream);

/*
 * Runs split over ranks (cube_params.nslab > 1).  The reference decomposes the box into
 * nn^3 images that exchange ncb-deep ghost layers of particles (buffer_particle.f90:29-375,
 * buffer_x / buffer_v in main.f90:36-38), transpose PM1 pencils (pencil_fft.f90:81-325) and
 * reduce the dt criteria over images (kick.f90:316-346).  Here the box is split along z
 * into nslab slabs of whole tile layers, one rank each.  A rank holds its own particles
 * plus ghost copies of the ncb coarse-cell layers next to its slab (refreshed before each
 * drift and each kick), runs PM2, PM3 and PP on its own tiles, drifts its own and ghost
 * particles and keeps the ones that land in its slab, and reduces the PM1 density over
 * ranks before a replicated PM1 solve.  With CUBE_DEPOSIT_FIXED every rank's particles end
 * up bit-identical to the nslab = 1 run of the whole box (integer sums do not depend on
 * their order); cube_step_out holds the global reductions on every rank (maxima, and sums
 * of pairs, masses and momentum; nplocal and napm stay per rank).
 *
 * The host supplies the two collectives through cube_comm (MPI, NCCL through
 * torch.distributed, ...).  Every rank makes the same library calls in the same order, so
 * the collectives match; a callback returning non-zero fails the call with CUBE_E_COMM.
 *  allreduce: in place over all ranks, `count` elements of `dtype` (CUBE_DT_*) with `op`
 *    (CUBE_OP_*).  device = 1: `buf` is device memory of the context's GPU (the library
 *    has synchronised its stream and reads the result when the call returns); 0: host.
 *  sendrecv: with the slab below (slab-1 mod nslab) and the slab above (slab+1 mod nslab):
 *    send `up` (sn_up bytes) to the slab above and `down` to the slab below; receive into
 *    `from_below` what the slab below sent up (rn_below bytes) and into `from_above` what
 *    the slab above sent down.  Sizes agree pairwise (the library exchanges them first);
 *    a zero-byte message may be skipped by both sides.  With nslab = 2 both neighbours
 *    are one rank: post the sends in the order up, down and the receives in the order
 *    from_below, from_above, so that messages pair up in order.
 * cube_gpu_set_comm copies the struct; it must be set before the first drift or kick of a
 * run with nslab > 1.  Such runs step eagerly (cube_params.step_graph is ignored), and
 * cube_gpu_ic and cube_gpu_power do not take them.  Upload and download carry the rank's
 * own particles: rhoc is the global array with zeros outside the slab.
 */
#define CUBE_DT_F32 0
#define CUBE_DT_I64 1
#define CUBE_DT_F64 2
#define CUBE_DT_I32 3
#define CUBE_OP_SUM 0
#define CUBE_OP_MAX 1
typedef struct cube_comm {
  void* user;
  int (*allreduce)(void* user, void* buf, int64_t count, int32_t dtype, int32_t op, int32_t device);
  int (*sendrecv)(void* user, const void* up, int64_t sn_up, const void* down, int64_t sn_down,
                  void* from_below, int64_t rn_below, void* from_above, int64_t rn_above,
                  int32_t device);
} cube_comm;
int cube_gpu_set_comm(cube_ctx* ctx, const cube_comm* comm);

/* Coarse-cell sets of slab p->slab of p->nslab as global storage indices of rhoc (the
 * order above), ascending; host arithmetic only, no device needed.  which: 0 the slab's
 * own cells, 1 the layer it sends down (its lowest ncb cell layers), 2 the layer it sends
 * up (its highest ncb), 3 its ghost layer from below (the slab below's highest ncb
 * layers), 4 its ghost layer from above.  Writes at most n indices (out may be NULL) and
 * returns the size of the set, or a negative CUBE_E_* code. */
int64_t cube_slab_cells(const cube_params* p, int which, int64_t* out, int64_t n);

/*
 * Differentiable particle-mesh step, for the adjoint (the PyTorch binding
 * cube_nu_b200/adjoint.py wraps it in torch.autograd.Function).  One periodic PM level on
 * an n^3 mesh in fine-cell units with the reference's PM pieces: TSC mass assignment
 * (particle_mesh.f90:56-62), the Green table of Green/Green.f90 with softening `soft` and
 * no range cut, the 4-point gradient (particle_mesh.f90:224-247), TSC interpolation, and
 * the KDK order of main.f90 (drift by D, then kick by K times the force).  Positions are
 * real numbers (not ZIPX codes) so that the step is differentiable.  All arrays are device
 * pointers on the context's device: x, v, u, gx are (np,3) floats, x in [0, n); rho and
 * lam are n^3 floats, x fastest.  Each call returns when its work is done.
 *   cube_dpm_kdk:         x += D v (wrapped), then v += K F(x)
 *   cube_dpm_force:       f = F(x)
 *   cube_dpm_force_vjp:   gx += d(sum_i u_i . F_i(x)) / dx   (the hand-written adjoint)
 *   cube_dpm_density:     rho = mass * sum_i W(x_i - c)
 *   cube_dpm_density_vjp: gx += d(sum_c lam(c) rho(c)) / dx
 *   cube_dpm_green:       the Green table, n*n*(n/2+1) floats [kz][ky][kx]
 */
typedef struct cube_dpm cube_dpm;
int cube_dpm_create(int n, float soft, float mass, int device, cube_dpm** out);
int cube_dpm_destroy(cube_dpm* d);
int cube_dpm_drift(cube_dpm* d, float* x, const float* v, int64_t np, float D);
int cube_dpm_kdk(cube_dpm* d, float* x, float* v, int64_t np, float D, float K);
int cube_dpm_force(cube_dpm* d, const float* x, int64_t np, float* f);
int cube_dpm_force_vjp(cube_dpm* d, const float* x, int64_t np, const float* u, float* gx);
int cube_dpm_density(cube_dpm* d, const float* x, int64_t np, float* rho);
int cube_dpm_density_vjp(cube_dpm* d, const float* x, int64_t np, const float* lam, float* gx);
int cube_dpm_green(cube_dpm* d, float* out, int64_t nout);

/* Text of the last error on this thread. */
int cube_gpu_last_error(char* buf, size_t n);
/* Library build string. */
const char* cube_gpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* CUBE_GPU_H */
