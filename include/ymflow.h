/*
 * ymflow — C ABI of the B200 Wilson gradient-flow engine (libymflow.so).
 *
 * Drop-in for the hot path of the reference's FLOW application
 * (GioPede/LatticeYangMills): the RK3 flow step, the Wilson force, the SU(3)
 * exponential and the plaquette / clover energy / clover charge observables.
 * Every entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Plain C types only; every call returns int status (0 = ok, < 0 = error)
 *     except the constructors, which return a handle and write the status.
 *   - Host buffers are caller-owned; device memory, streams and graphs belong
 *     to the context.  One context per host thread: calls on one context are
 *     not reentrant; separate contexts are independent (one CUDA stream each).
 *   - Links on the host use the reference's .bin layout
 *     (src/InputOutput/inputconf.cpp:114-155): site-major with x fastest,
 *     site = x + Nx*(y + Ny*(z + Nz*t)), then mu = 0..3, then 18 doubles per
 *     link, a row-major 3x3 complex matrix with (re, im) interleaved
 *     (include/Math/su3.h:63).
 *   - No call exits or aborts the process; the text of the last error is
 *     available from ymflow_last_error().
 */
#ifndef YMFLOW_H
#define YMFLOW_H

#include <stdint.h>

#if defined(__GNUC__)
#define YMFLOW_API __attribute__((visibility("default")))
#else
#define YMFLOW_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------- */
#define YMFLOW_OK 0
#define YMFLOW_ERR_ARG (-1)         /* bad argument (null pointer, size, precision ...) */
#define YMFLOW_ERR_CUDA (-2)        /* a CUDA call failed; see ymflow_last_error */
#define YMFLOW_ERR_OOM (-3)         /* device or pinned host allocation failed */
#define YMFLOW_ERR_NONFINITE (-4)   /* a measured observable was NaN or infinite */
#define YMFLOW_ERR_UNITARITY (-5)   /* mixed path: links drifted from SU(3) beyond the limit */
#define YMFLOW_ERR_CAPACITY (-6)    /* caller's output array too small */
#define YMFLOW_ERR_STATE (-7)       /* call out of order (e.g. flow before upload) */
#define YMFLOW_ERR_NODEVICE (-8)    /* no CUDA device, or the device is not sm_100 */

/* ---- precisions ------------------------------------------------------------------- */
#define YMFLOW_FP64 0     /* FP64 links (18 reals), FP64 arithmetic: the parity path */
#define YMFLOW_FP32_18 1  /* FP32 links (18 reals) and site arithmetic, FP64 reductions */
#define YMFLOW_FP32_12 2  /* FP32 two-row links (12 reals, third row rebuilt), FP64 reductions */

/* ---- seeded synthetic fields (ymflow_init_links) ------------------------------------ */
#define YMFLOW_FIELD_COLD 0    /* every link the identity */
#define YMFLOW_FIELD_EXPIAH 1  /* U = e^{i a H}, H traceless Hermitian, iid N(0,1) reals */
#define YMFLOW_FIELD_HOT 2     /* (ymflow_generate_metropolis start) Haar-random links */
#define YMFLOW_FIELD_CURRENT 3 /* (ymflow_generate_metropolis start) continue from the current links */

typedef struct ymflow_ctx ymflow_ctx;

/* One measurement: the reference's SuperObs public fields
 * (include/Observables/observable.h:60) plus the flow time and t^2 <E>. */
typedef struct {
    int32_t step;   /* flow steps taken before this measurement */
    int32_t pad;
    double t;       /* flow time, accumulated as t += eps (src/Apps/wilsonflow.cpp:126) */
    double plaq;    /* SuperObs::plaq   = sum Re tr P / (18 V)               (superobs.cpp:125) */
    double topc;    /* SuperObs::topc   = -sum Re tr(G G~) / (256 pi^2)      (superobs.cpp:114-126) */
    double energy;  /* SuperObs::energy = sum Re tr(G G), raw clover sum     (superobs.cpp:109) */
    double t2E;     /* t^2 <E> = -t^2 energy / (64 V) */
} ymflow_obs;

/* Library version string (no counterpart in the reference). */
YMFLOW_API const char* ymflow_version(void);

/* Number of usable (sm_100) CUDA devices; the reference's rank count comes from
 * MPI instead (src/ParallelTools/parallel.cpp:57-70). */
YMFLOW_API int ymflow_device_count(int* count);

/* Create a flow context for a dims[0] x dims[1] x dims[2] x dims[3] periodic
 * lattice (x, y, z, t) on `device`.  Replaces WilsonFlow::createLattice
 * (src/Apps/wilsonflow.cpp:87-91), which allocates the GluonField and the
 * force field, and PureGauge's scratch fields (src/Actions/puregauge.cpp:18-25). */
YMFLOW_API ymflow_ctx* ymflow_create(const int dims[4], int precision, int device, int* status);

/* Release every device resource of the context.  NULL is accepted. */
YMFLOW_API void ymflow_destroy(ymflow_ctx* ctx);

/* Text of the last error on this context (never NULL).  With ctx == NULL:
 * the last error of a failed ymflow_create. */
YMFLOW_API const char* ymflow_last_error(const ymflow_ctx* ctx);

/* Load links from a host buffer in .bin layout (4*V*18 doubles).
 * Replaces LatticeIO::InputConf::readConf's fill of the GluonField
 * (src/InputOutput/inputconf.cpp:114-155). */
YMFLOW_API int ymflow_upload(ymflow_ctx* ctx, const double* links_aos);

/* Store the current links to a host buffer in .bin layout (4*V*18 doubles).
 * (The reference's writer is a no-op, src/InputOutput/outputconf.cpp:102.) */
YMFLOW_API int ymflow_download(ymflow_ctx* ctx, double* links_aos);

/* Ranged transfers for large lattices: sites [first_site, first_site + nsites)
 * in the .bin layout (links_aos points at site first_site's first double), so a
 * caller can stream a configuration file through a small (ideally pinned,
 * ymflow_host_alloc) buffer instead of holding the whole field in host memory.
 * flags: YMFLOW_IO_BIG_ENDIAN = every double byte-reversed, the big-endian
 * ("Chroma") files of the reference's commented reader variant
 * (src/InputOutput/inputconf.cpp:135-143); the reversal runs on the device.
 * An upload marks the field loaded and resets the flow time; the caller covers
 * every site before flowing.  Synchronous like ymflow_upload/ymflow_download;
 * the device staging buffer grows to the largest range used. */
#define YMFLOW_IO_BIG_ENDIAN 1

/* Load a .bin configuration file into the context (its part of it, for a
 * slab): the file is read in chunks of chunk_sites sites (0: 65536) through two
 * pinned buffers, the read of one chunk overlapping the copy and unpacking of
 * the one before, so a 64^4 file (9.7 GB) loads at disk speed with no
 * whole-field host copy.  flags as for ymflow_upload_sites; YMFLOW_ERR_ARG if
 * the file's size is not the configuration's. */
YMFLOW_API int ymflow_load_file(ymflow_ctx* ctx, const char* path, int flags, int64_t chunk_sites);
YMFLOW_API int ymflow_upload_sites(ymflow_ctx* ctx, const double* links_aos, int64_t first_site, int64_t nsites,
                                   int flags);
YMFLOW_API int ymflow_download_sites(ymflow_ctx* ctx, double* links_aos, int64_t first_site, int64_t nsites,
                                     int flags);

/* Fill the links with a seeded synthetic field on the device: kind COLD or
 * EXPIAH (scale a); then, if haar_frac > 0, replace that fraction of links
 * (seeded Bernoulli) by Haar-random SU(3).  Same recipe as the test fixtures. */
YMFLOW_API int ymflow_init_links(ymflow_ctx* ctx, int kind, double a, uint64_t seed, uint32_t config, double haar_frac);

/* Generate a configuration by Metropolis updates of the Wilson action at
 * `beta`: `sweeps` sweeps, each a checkerboard over (mu, site parity), `hits`
 * proposals X U per link with X a product of three SU(2) elements of size
 * `su3eps` (or X^+ U, with probability 1/2, so the proposal is symmetric),
 * accepted when exp(-dS) > r with dS = -(beta/3) Re tr[(U' - U) A].
 * Starts from a cold, hot (Haar) or the current field.  Seeded and
 * reproducible (counter-based Philox per link, sweep and hit); sweeps are
 * numbered from the last cold/hot start, so a CURRENT call continues the
 * chain (two calls of n sweeps equal one of 2n with the same seed).  Replaces the
 * reference's GaugeFieldFactory update (src/Apps/gaugefieldfactory.cpp:192-220,
 * src/Math/random.cpp:71-156), whose source does not compile.  FP32 forms are
 * reunitarised in FP64 after every sweep.  *acceptance (optional) receives the
 * accepted fraction.  Every extent must be even (YMFLOW_ERR_ARG otherwise). */
YMFLOW_API int ymflow_generate_metropolis(ymflow_ctx* ctx, int start, double beta, double su3eps, int sweeps,
                                          int hits, uint64_t seed, double* acceptance);

/* Plaquette, clover energy and clover charge of the current links.
 * Replaces SuperObs::compute (src/Observables/superobs.cpp:31-128) including
 * its MPI_Allreduce (:24-28).  out->step / out->t are the context's counters. */
YMFLOW_API int ymflow_observables(ymflow_ctx* ctx, ymflow_obs* out);

/* Flow nsteps Luscher RK3 steps of size eps (WilsonFlow::flowStep,
 * src/Apps/wilsonflow.cpp:141-172).  A measurement is taken before the first
 * step (row 0, as src/Apps/wilsonflow.cpp:120-123), after every
 * `measure_every`-th step and after the last step; measure_every <= 0 measures
 * only before and after.  Mixed precisions reunitarise in FP64 every
 * `reunit_every` steps (<= 0: never; the FP64 path ignores it, as the
 * reference never reunitarises).  Rows go to out[0 .. *n_out-1]; out_cap must
 * hold them all (YMFLOW_ERR_CAPACITY otherwise, before any work).  Returns
 * YMFLOW_ERR_NONFINITE if a measurement is NaN/inf, YMFLOW_ERR_UNITARITY if a
 * reunitarisation saw a row norm off by more than 1e-3. */
YMFLOW_API int ymflow_flow(ymflow_ctx* ctx, double eps, int nsteps, int measure_every, int reunit_every, ymflow_obs* out,
                int out_cap, int* n_out);

/* The flow generator Z_mu(x) = (i/2)[U Omega - (U Omega)^+]_traceless of the
 * current links for one direction mu, as V full 3x3 Hermitian matrices (18
 * doubles each, site order).  Replaces PureGauge::computeDerivative(mu)
 * (src/Actions/puregauge.cpp:62-79; staples :36-54). */
YMFLOW_API int ymflow_derivative(ymflow_ctx* ctx, int mu, double* z_host);

/* e^{iQ} of n Hermitian traceless 3x3 matrices (18 doubles each, only the
 * diagonal entries 0 and 1 and the upper triangle are read) on `device`.
 * Replaces exp(const SU3&) (src/Math/su3.cpp:96-183); where that returns NaN
 * (Q = 0, or rounding past acos's domain on a degenerate spectrum) this
 * returns the exponential. */
YMFLOW_API int ymflow_su3_exp(const double* q_host, double* r_host, int64_t n, int device);

/* Reset the context's step and flow-time counters (a new configuration). */
YMFLOW_API int ymflow_reset_time(ymflow_ctx* ctx);

/* Set the step and flow-time counters, to resume a flow from a checkpoint:
 * ymflow_download the links and keep the last row's (step, t); later
 * ymflow_upload them and set (step, t) to continue with the same rows as an
 * unbroken flow (the reference keeps no flow checkpoint; its configuration
 * writer is a no-op, src/InputOutput/outputconf.cpp:102). */
YMFLOW_API int ymflow_set_time(ymflow_ctx* ctx, int64_t step, double t);

/* Device-timed flow steps for benchmarking: runs nsteps RK3 steps (no
 * measurements) between two CUDA events on the context's stream and writes the
 * elapsed milliseconds.  kernel_ms (optional, may be NULL) receives the summed
 * duration of the stage kernels alone, timed with events around each launch. */
YMFLOW_API int ymflow_time_steps(ymflow_ctx* ctx, double eps, int nsteps, float* elapsed_ms, float* kernel_ms);

/* The same with the kernels of the two-kernel stage (YMFLOW_OPT_STAGE_FORM 1)
 * timed apart: field_ms (optional) receives the summed duration of the
 * plaquette-field kernels (0 for the fused form), stage_ms (optional) that of
 * the stage kernels, each from events around every launch. */
YMFLOW_API int ymflow_time_kernels(ymflow_ctx* ctx, double eps, int nsteps, float* elapsed_ms, float* field_ms,
                                   float* stage_ms);

/* Tuning knobs.  key YMFLOW_OPT_BLOCK: threads per block of the stage kernel
 * (128: four warps, one per direction, per 32 sites); YMFLOW_OPT_OBS_BLOCK:
 * threads per block of the observables kernel (192: six warps, one per
 * plane, per 32 sites; read-only in effect, other values are rejected);
 * YMFLOW_OPT_GRAPH: 1 = replay each RK3 step as a captured CUDA graph
 * (default), 0 = plain launches; YMFLOW_OPT_STAGE_FORM: the kernels of one RK3
 * stage (the reference's computeDerivative + exp + link update for all mu,
 * src/Apps/wilsonflow.cpp:143-171):
 *   0 = one fused kernel, staples summed per link (the FP64 default where
 *       form 1's field does not fit in device memory);
 *   1 = two kernels, the six plaquettes' generators of every site into a
 *       stored field (6 x 8 reals per site of device memory), then each link's
 *       force from them (the default, except FP32 lattices of at most 8192
 *       sites, whose launch-bound steps run form 0);
 *   2 = one kernel: blocks of Lx x ty x tz sites of a time slice compute their
 *       plaquette generators into shared memory, recompute the lower (y, z)
 *       faces, stream along t and finish the links from there (whole-lattice
 *       contexts only; ymflow_autotune times it against the others).
 * YMFLOW_OPT_TILE: form 2's tiling, value = (lean << 36) | (lpt << 32) |
 * (ty << 16) | tz: ty must divide the y extent, tz the z extent, Lx ty must be
 * a multiple of 32 and Lx ty tz within 64..512 sites; each thread advances
 * lpt = 1, 2 or 4 links (0 reads as 4), so a block has 4 Lx ty tz / lpt
 * threads; lean = 1 runs the kernel compiled for 64 registers (up to 1024
 * threads), lean = 0 the one for 128 (up to 512).  YMFLOW_ERR_ARG otherwise.  YMFLOW_OPT_TIMED_REUNIT: the FP64
 * reunitarisation of the mixed forms after every n-th step of
 * ymflow_time_steps / ymflow_time_kernels (0 = none, the default), so timed
 * steps can carry it as ymflow_flow's reunit_every does.
 * Slabs flowing together (ymflow_slab_group_flow) must share one form. */
#define YMFLOW_OPT_BLOCK 1
#define YMFLOW_OPT_GRAPH 2
#define YMFLOW_OPT_OBS_BLOCK 3
#define YMFLOW_OPT_STAGE_FORM 4
#define YMFLOW_OPT_TILE 5
#define YMFLOW_OPT_TIMED_REUNIT 6
YMFLOW_API int ymflow_set_option(ymflow_ctx* ctx, int key, int64_t value);
YMFLOW_API int ymflow_get_option(const ymflow_ctx* ctx, int key, int64_t* value);

/* The project's autotuner for one context (no counterpart in the reference,
 * whose stage is a fixed sequence of whole-lattice passes,
 * src/Apps/wilsonflow.cpp:141-172): times one RK3 stage in every form and
 * tiling the lattice allows (form 0, form 1, form 2 at every valid (ty, tz)),
 * keeps the fastest, and caches the choice for every context of the same
 * extents, precision and device in the process.  The current links are not
 * changed (stage 0 runs into the other buffer).  Forms agree to rounding, so
 * a tuned flow can differ from the default one in the last bits.  Writes the
 * chosen form and tile (0, 0 unless form 2).  Not for slab contexts. */
YMFLOW_API int ymflow_autotune(ymflow_ctx* ctx, double eps, int* stage_form, int* tile_y, int* tile_z);

/* --- One configuration split along t over several GPUs -------------------- */
/* A slab context holds the time slices [t0, t0 + nt) of a configuration of
 * extents global_dims on one GPU, with one halo slice on each side.  It
 * replaces the reference's MPI domain decomposition
 * (src/ParallelTools/parallel.cpp:57-100, "SubLatticeSize") for the time
 * direction.  The spatial volume x y z must be a multiple of 32.
 * ymflow_upload/_download/_upload_sites/_download_sites address the slab's own
 * sites, which are sites [t0 Vs, (t0 + nt) Vs) of the .bin file (Vs = x y z).
 * ymflow_init_links draws the same links as a whole-lattice context with the
 * same seed.  Observables are of the whole configuration once summed over the
 * slabs.  ymflow_derivative and ymflow_generate_metropolis need a whole-lattice
 * context.
 *
 * A slab flows in one of two ways:
 *  - one process per GPU: ymflow_slab_connect, then ymflow_flow /
 *    ymflow_observables / ymflow_time_steps as usual.  These become collective
 *    over the ranks (every rank calls them with the same arguments).  Halos
 *    travel by NCCL send/recv after every stage; measurement rows are summed
 *    with an NCCL all-reduce.  NCCL is loaded at run time: the library named
 *    by YMFLOW_NCCL_LIB, else a libnccl.so.2 the process already holds, else
 *    the loader's libnccl.so.2 (a process must hold one NCCL: set
 *    YMFLOW_NCCL_LIB to a framework's copy if that framework is imported
 *    later); YMFLOW_ERR_NODEVICE if none loads.
 *  - several slabs in one process (one or more GPUs): ymflow_slab_group_flow,
 *    with halos as stream-ordered peer copies.
 * A slab that is neither connected nor flowed through its group returns
 * YMFLOW_ERR_STATE from ymflow_flow. */
YMFLOW_API ymflow_ctx* ymflow_create_slab(const int global_dims[4], int t0, int nt, int precision, int device,
                                          int* status);

/* NCCL communicator set-up, in place of the reference's MPI Cartesian
 * communicator and neighbour ranks (src/ParallelTools/parallel.cpp:72-100):
 * rank 0 makes the id and shares its bytes with the other ranks (e.g. through
 * torch.distributed); every rank then connects its slab, naming the ranks that
 * hold the slices below t0 and above t0 + nt - 1 (periodically; a single rank
 * is its own neighbour). */
#define YMFLOW_NCCL_ID_BYTES 128
YMFLOW_API int ymflow_nccl_unique_id(void* id);
YMFLOW_API int ymflow_slab_connect(ymflow_ctx* ctx, const void* id, int rank, int nranks, int lower_rank,
                                   int upper_rank);

/* ymflow_flow over the n slab contexts of one configuration, in time order
 * (ctxs[i] starts where ctxs[i-1] ends), held in this process: the reference's
 * flow on a decomposed lattice (WilsonFlow::flowStep with shift()'s face
 * exchange, src/Apps/wilsonflow.cpp:141-172, include/Math/lattice.h:437-449).
 * Rows as ymflow_flow's, for the whole configuration. */
YMFLOW_API int ymflow_slab_group_flow(ymflow_ctx* const* ctxs, int n, double eps, int nsteps, int measure_every,
                                      int reunit_every, ymflow_obs* out, int out_cap, int* n_out);

/* --- One configuration split in any set of directions (blocks) ---------- */
/* A block context holds the sites [origin, origin + extent) of a configuration
 * of extents global_dims (extent = global in a direction the decomposition
 * does not split) in a local lattice with one halo layer on each side of every
 * split direction.  It replaces the reference's Cartesian domain decomposition
 * in full (src/ParallelTools/parallel.cpp:57-100, SubLatticeSize in any
 * direction, with the second-neighbour exchange of the clover, :117-140) for
 * the blocks of one process on one or several GPUs.  ymflow_upload /
 * ymflow_download / _sites address the block's own sites in lexicographic
 * order over its extents (.bin layout); ymflow_init_links, ymflow_load_file,
 * ymflow_flow and ymflow_observables of a single block return an error
 * (flow and measure the group). */
YMFLOW_API ymflow_ctx* ymflow_create_block(const int global_dims[4], const int origin[4], const int extent[4],
                                           int precision, int device, int* status);

/* ymflow_flow over the n = grid[0] grid[1] grid[2] grid[3] blocks of one
 * configuration held in this process, ctxs[i] at grid coordinates
 * (i % grid[0], i / grid[0] % grid[1], ...) with origins increasing along each
 * direction; blocks on different GPUs must reach each other's memory.  After
 * every stage each block pulls its halos from its neighbours, one split
 * direction at a time, which also fills the edges the staples and the clover
 * read.  Rows as ymflow_flow's, for the whole configuration. */
YMFLOW_API int ymflow_block_group_flow(ymflow_ctx* const* ctxs, int n, const int grid[4], double eps, int nsteps,
                                       int measure_every, int reunit_every, ymflow_obs* out, int out_cap,
                                       int* n_out);

/* Measured CUDA-core FMA throughput of `device` in TFLOP/s (2 flops per FMA):
 * FP64 FMAs for YMFLOW_FP64, FP32 FMAs otherwise.  A measurement utility with
 * no counterpart in the reference: the denominator of the stage kernels'
 * arithmetic roofline.  Runs twelve short kernels (about 0.1 s); best of eleven. */
YMFLOW_API int ymflow_fma_peak(int device, int precision, double* tflops);

/* Page-locked host memory for transfers at full PCIe rate (cudaMallocHost). */
YMFLOW_API int ymflow_host_alloc(int64_t bytes, void** ptr);
YMFLOW_API int ymflow_host_free(void* ptr);

/* Device bytes held by the context (links x2, force, staging, scratch). */
YMFLOW_API int ymflow_device_bytes(const ymflow_ctx* ctx, int64_t* bytes);

/* ---- allocation-free observables ----------------------------------------------------
 * No counterpart in the reference: an extra entry point for callers that cannot
 * call cudaMalloc where they measure, e.g. a host application that reserved the
 * whole device for its own memory pool, or a latency-critical loop that cannot
 * take the implicit synchronisation of an allocation.
 *
 * Computes plaq, topc and energy (as ymflow_observables) of a configuration the
 * caller holds in DEVICE memory in the .bin layout (4*V*18 doubles, FP64) and
 * writes out_device[0..3] = plaq, topc, energy, non-finite flag (0 or 1), in
 * device memory, asynchronously on `stream` (a cudaStream_t; NULL = default
 * stream) of the current device.  Allocates nothing: its scratch is a fixed
 * 1.5 MB device array inside the library (held by every GPU that loads it),
 * which limits the lattice to YMFLOW_NOALLOC_MAX_SITES sites; larger lattices
 * return YMFLOW_ERR_CAPACITY.  links_aos_device must be 16-byte aligned and
 * out_device 8-byte aligned (YMFLOW_ERR_ARG otherwise, before any launch).
 * The first call on a device looks the array's device address up once and
 * should come before any stream capture; the cached address does not survive
 * a cudaDeviceReset.  All calls share the array: calls that overlap on the GPU
 * race and must be ordered by the caller.  Returns YMFLOW_ERR_ARG,
 * YMFLOW_ERR_CAPACITY, YMFLOW_ERR_NODEVICE or YMFLOW_ERR_CUDA (launch failure)
 * on error. */
#define YMFLOW_NOALLOC_MAX_SITES 8388608
YMFLOW_API int ymflow_observables_noalloc(const double* links_aos_device, const int dims[4], double* out_device,
                                          void* stream);

/* ---- batched ensemble --------------------------------------------------------------
 * Many configurations, of any mix of lattice sizes, flowed together: every RK3
 * stage of every configuration is one persistent launch over a work list of
 * (configuration, block of sites), and each step is replayed as a captured CUDA
 * graph.  Replaces the reference's one-by-one loop over the sorted InputDir
 * files (src/Apps/wilsonflow.cpp:96-109).  Output rows are [row][conf]. */
typedef struct ymflow_ens ymflow_ens;

/* dims: nconf x 4 extents (x, y, z, t) per configuration. */
YMFLOW_API ymflow_ens* ymflow_ensemble_create(int nconf, const int* dims, int precision, int device, int* status);
YMFLOW_API void ymflow_ensemble_destroy(ymflow_ens* ens);
YMFLOW_API const char* ymflow_ensemble_last_error(const ymflow_ens* ens);
YMFLOW_API int ymflow_ensemble_upload(ymflow_ens* ens, int conf, const double* links_aos);
YMFLOW_API int ymflow_ensemble_download(ymflow_ens* ens, int conf, double* links_aos);
YMFLOW_API int ymflow_ensemble_init_links(ymflow_ens* ens, int conf, int kind, double a, uint64_t seed,
                                          uint32_t config, double haar_frac);
/* As ymflow_flow for every configuration at once; out holds rows_cap x nconf entries. */
YMFLOW_API int ymflow_ensemble_flow(ymflow_ens* ens, double eps, int nsteps, int measure_every, int reunit_every,
                                    ymflow_obs* out, int rows_cap, int* n_rows);
YMFLOW_API int ymflow_ensemble_reset_time(ymflow_ens* ens);
/* Device-timed RK3 steps of the whole ensemble (no measurements). */
YMFLOW_API int ymflow_ensemble_time_steps(ymflow_ens* ens, double eps, int nsteps, float* elapsed_ms);
/* The project's autotuner for an ensemble: times one RK3 stage of the whole
 * ensemble in each form it can take and keeps the fastest, cached for every
 * ensemble of the same sizes and precision in the process:
 *   - the per-link kernel (FP64) over persistent grids {one CTA per work
 *     item, 1x and 2x the resident CTAs}, or the two-kernel stage (FP32), one
 *     block per 32-site item;
 *   - the two-kernel stage launched once per run of consecutive
 *     configurations with equal extents, each run's geometry a launch
 *     parameter (two launches per run and stage; FP64 ensembles where their
 *     plane-generator pool fits);
 *   - the one-kernel stage with tiles in shared memory (YMFLOW_OPT_STAGE_FORM
 *     2 of a single context) at 128, 256, 384 or 512 threads per block: every
 *     configuration gets the tile of at most that many sites (whole x lines,
 *     a ty x tz patch of (y, z)) with the least estimated time per site, and
 *     one persistent launch per stage streams along t through the tile units
 *     of all configurations.
 * Writes the block size and grid of the choice (grid 0: one block per item).
 * Does not change the flow state. */
YMFLOW_API int ymflow_ensemble_autotune(ymflow_ens* ens, double eps, int* block, int* grid);
/* The ensemble's current stage form (0 per-link kernel, 1 two-kernel stage,
 * 2 tiles in shared memory, 3 two-kernel stage per run of equal extents),
 * block size and grid. */
YMFLOW_API int ymflow_ensemble_tuning(const ymflow_ens* ens, int* stage_form, int* block, int* grid);
/* Sets the form by hand: 0 with block 128 and a grid (0: one block per item),
 * 1 or 3 with block 128 (ensembles with a plane-generator pool: every FP32
 * one, FP64 ones where it fits), or 2 with `block` threads (grid chosen from
 * the occupancy).  YMFLOW_ERR_ARG where the form cannot run. */
YMFLOW_API int ymflow_ensemble_set_tuning(ymflow_ens* ens, int stage_form, int block, int grid);

#ifdef __cplusplus
}
#endif
#endif /* YMFLOW_H */
