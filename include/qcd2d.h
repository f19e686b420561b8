/*
 * qcd2d.h — C ABI of the B200-native checkerboard SU(2) Wilson-action sweep.
 *
 * Drop-in for the hot path of fezquerro/QCD_2d_GPU (2+1-D SU(2) lattice gauge
 * theory, links stored as unit quaternions).  The reference has no library
 * boundary: its host program kernel.cu calls device-buffer launchers
 * (`mc_up_per/pcc/pmc`, `normalize`, `en_av`, `setup_kernel`, the init
 * kernels) directly from main().  Each entry point below replaces one of those
 * call sites; the citation on each declaration names it (file:line of the
 * reference).  Device memory is owned by the library, host buffers by the
 * caller.  One lattice handle = one CUDA stream; a handle is not thread-safe.
 * Every function returns QCD_OK (0) or a negative qcd_status; the message of
 * the last failure on a handle is qcd_last_error(h).
 *
 * Layout at the boundary (qcd_load_config / qcd_store_config) is the
 * reference's: V*12 doubles, site-major, even sublattice first
 * (site = id for even sites, id + V/2 for odd sites, id = y' + (Ly/2)*(x + Lx*t)),
 * 3 links per site in the order y, x, t, 4 quaternion components each
 * (kernel.cu:58, lattice_setup.h:24-37, output.h:77-94).
 */
#ifndef QCD2D_H
#define QCD2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
enum qcd_status {
  QCD_OK = 0,
  QCD_ERR_INVALID = -1,     /* bad argument: odd or zero size, bad enum, null pointer */
  QCD_ERR_CUDA = -2,        /* a CUDA runtime call failed (message in qcd_last_error) */
  QCD_ERR_NOMEM = -3,       /* device allocation failed */
  QCD_ERR_NONUNITARY = -4,  /* a link's determinant is far from 1 or not finite */
  QCD_ERR_TIMEOUT = -5,     /* a bounded device-side wait ran out */
  QCD_ERR_IO = -6,          /* configuration file missing, short or malformed */
  QCD_ERR_UNSUPPORTED = -7  /* combination not provided (e.g. FP32 Metropolis in parity mode) */
};

/* update algorithm: values of kernel.cu:11-12 (METROPOLIS 0, HEATBATH 1) */
enum qcd_algo { QCD_ALGO_METROPOLIS = 0, QCD_ALGO_HEATBATH = 1 };

/* y boundary condition: values of kernel.cu:28 (Boundary) */
enum qcd_boundary { QCD_BC_PERIODIC = 0, QCD_BC_PCC = 1, QCD_BC_PMC = 2 };

/* link storage / arithmetic */
enum qcd_precision {
  /* FP64 links and the reference's exact operation order and RNG draw order:
     reproduces the reference link field (max|dU| <= 1e-12 after 10 sweeps) */
  QCD_PREC_FP64 = 0,
  /* FP32 links and FP32 staples / heat-bath / over-relaxation; FP64 kept for the
     Kennedy-Pendleton a0 near 1, the Metropolis exact fallback, link
     re-projection and the global plaquette/energy sums */
  QCD_PREC_FP32 = 1
};

/* Parameters of one lattice.  Mirrors `struct lattice` (lattice_setup.h:2-14)
   and the #define knobs of kernel.cu:11-46 that concern the sweep. */
typedef struct qcd_params {
  int lt, lx, ly;          /* d_t, d_x, d_y (kernel.cu:24-26); all even and >= 2 */
  float beta;              /* betal (kernel.cu:27); float like lattice.beta */
  float epsilon;           /* epsilonl (kernel.cu:43), Metropolis proposal size */
  int upd;                 /* upd (kernel.cu:44), Metropolis hits per link */
  int algo;                /* enum qcd_algo (kernel.cu:13) */
  int boundary;            /* enum qcd_boundary (kernel.cu:28) */
  int precision;           /* enum qcd_precision */
  int n_or;                /* over-relaxation passes after each heat-bath/Metropolis
                              pass inside qcd_sweep (0 = the reference's sweep) */
  int renorm_every;        /* re-project all links every this many qcd_sweep sweeps
                              (0 = never inside qcd_sweep; the host calls
                              qcd_normalize, as kernel.cu:163,203 does) */
  unsigned long long seed; /* seed of the MRG32k3a streams (lattice_setup.h:15-21) */
} qcd_params;

typedef struct qcd_lattice qcd_lattice;

/* Fill p with the reference's defaults for an Lt x Lx x Ly lattice. */
void qcd_params_default(qcd_params* p, int lt, int lx, int ly);

/* Allocate the link store, the V/2 MRG32k3a streams (curand_init(seed, id, 0),
   replaces setup_kernel, kernel.cu:77-79 / lattice_setup.h:15-21) and the
   measurement buffers.  Rejects odd sizes like kernel.cu:61-64. */
int qcd_create(const qcd_params* p, qcd_lattice** out);
int qcd_destroy(qcd_lattice* h);

/* Launch everything on `stream` (a cudaStream_t); NULL restores the handle's
   own stream. */
int qcd_set_stream(qcd_lattice* h, void* stream);
/* The cudaStream_t the handle currently launches on. */
void* qcd_get_stream(qcd_lattice* h);

/* Cold start: all links = 1 (id_init2, lattice_setup.h:38-51; kernel.cu:94). */
int qcd_init_cold(qcd_lattice* h);
/* Hot start: 4 uniform doubles in (-0.5,0.5] per link, normalised, drawn from
   stream id in the order even y,x,t then odd y,x,t (rand_init2,
   lattice_setup.h:24-37); with PCC the x,t links at y=0 stay 1 and draw
   nothing (rand_init2_pcc, lattice_setup.h:52-81; kernel.cu:91,108,125). */
int qcd_init_hot(qcd_lattice* h);

/* Configuration in the reference's AoS FP64 layout (see top of file).
   Host buffers: read_conf + cudaMemcpy H2D (lattice_setup.h:83-100,
   kernel.cu:98-99) and cudaMemcpy D2H + save_conf (kernel.cu:183-185,
   output.h:77-94).  FP32 lattices convert at the boundary. */
int qcd_load_config(qcd_lattice* h, const double* aos_host);
int qcd_store_config(qcd_lattice* h, double* aos_host);
/* Same with device buffers of V*12 doubles (no host copy). */
int qcd_load_config_device(qcd_lattice* h, const double* aos_dev);
int qcd_store_config_device(qcd_lattice* h, double* aos_dev);

/* n full sweeps.  One sweep = the 6 checkerboard phases even_y, odd_y, even_x,
   odd_x, even_t, odd_t with heat-bath or `upd` Metropolis hits per link
   (mc_up_per mc_updates.h:467-475, mc_up_pcc mc_updates_pcc.h:216-224,
   mc_up_pmc mc_updates_pmc.h:249-257; called at kernel.cu:166-170,196-200),
   then n_or over-relaxation passes, then re-projection if renorm_every says so. */
int qcd_sweep(qcd_lattice* h, int n);
/* n over-relaxation passes over the 6 phases (mc_up_per(..., update=1),
   mc_updates.h:109-115,178-181; extended to PCC/PMC with the same masks). */
int qcd_overrelax(qcd_lattice* h, int n);
/* Re-project every link onto SU(2) (normalize, lattice_setup.h:202-207;
   kernel.cu:163-164,179,203-204). */
int qcd_normalize(qcd_lattice* h);

/* Energy = mean over sites of -(1 - P_xt) and average plaquette
   = mean of (P_yx + P_yt + P_xt)/3, PMC counting the y-plaquettes at
   y = Ly-1 as 1 (en_av<PMC>, observables.h:99-141; kernel.cu:208).
   FP64 sums in a fixed order: the result does not depend on scheduling.
   Synchronous: waits for the stream. */
int qcd_measure(qcd_lattice* h, double* energy, double* plaquette);
/* Asynchronous form: writes (energy, plaquette) into slot `index` of the
   handle's device series (capacity set by qcd_series_reserve); read the
   series back with qcd_series_read. */
int qcd_series_reserve(qcd_lattice* h, int capacity);
int qcd_measure_into_series(qcd_lattice* h, int index);
int qcd_series_read(qcd_lattice* h, double* energy, double* plaquette, int n);

/* Accepted updates per site since the last reset, V ints in the reference's
   site order (the `accept` array of kernel.cu:144-145, filled by
   link_update mc_updates.h:119-128 and read by mean_lattice,
   statistics.h:17-28).  Heat-bath and over-relaxation count 1 per link. */
int qcd_accept_counts(qcd_lattice* h, int* host_out);
int qcd_accept_reset(qcd_lattice* h);

/* Check that every link has |det - 1| <= tol and is finite; returns
   QCD_ERR_NONUNITARY otherwise (the device writes a flag, nothing traps).
   The mean determinant (print_det, lattice_setup.h:176-183) goes to *mean_det
   when it is not NULL. */
int qcd_check_unitarity(qcd_lattice* h, double tol, double* mean_det);

/* ------------------------------------------------------------------------
 * Scheduling of the six checkerboard phases (replaces the reference's six
 * serial launches per sweep, mc_updates.h:467-475, with the same result).
 *   PHASES     one launch per phase: each phase streams the link store.
 *   WAVEFRONT  one persistent launch per chain of passes: every t-slice goes
 *              through the phases of the chain while it is resident in L2;
 *              tasks run in a ring schedule ordered so that each waits only
 *              for earlier ones (bounded waits, QCD_ERR_TIMEOUT otherwise).
 *              Bit-identical to PHASES.
 *   PAIRS      FP32 only: each pass as three launches, one per direction mu,
 *              each fusing the phases (mu, even) and (mu, odd).  A CTA owns a
 *              tile of the plane perpendicular to its streamed direction and
 *              walks along it with the six link classes of the coming slices
 *              staged in shared memory by bulk asynchronous copies, so a link
 *              leaves HBM about once per pair instead of once per phase.  The
 *              pass writes its links into a second store (allocated when the
 *              schedule is set) that then becomes current.  Same updates and
 *              draws as PHASES; results agree with it to float rounding.
 *   AUTO       the schedule measured fastest for the lattice (currently PHASES).
 * ------------------------------------------------------------------------ */
enum qcd_schedule { QCD_SCHED_AUTO = 0, QCD_SCHED_PHASES = 1, QCD_SCHED_WAVEFRONT = 2, QCD_SCHED_PAIRS = 3 };
int qcd_set_schedule(qcd_lattice* h, int mode);
/* the schedule qcd_sweep will use (PHASES, WAVEFRONT or PAIRS) */
int qcd_get_schedule(const qcd_lattice* h);
/* FP32 store layout.  An FP32 lattice with Lt % 4 == 0 keeps its links in
   site pairs under the per-phase schedule: site id (t < Lt/2) and site
   id + V/4 (t + Lt/2) of a link class share one 32-B record (w0 w1 x0 x1)
   (y0 y1 z0 z1), and one thread updates both with packed two-lane FP32
   arithmetic (20-30% fewer instructions per link update; each quaternion
   product takes half).  Same updates
   and draws as one float4 plane per class; results agree with it to float
   rounding.  on = 0 keeps such a lattice on one float4 plane per class (the
   layout of the wavefront and fused-pair schedules and of the batched
   replicas, and the one those are bit-identical to); on = 1 (the default)
   allows the pairs.  The store is rewritten at once if the layout changes
   (values kept exactly).  Not a reference interface: the reference stores
   FP64 AoS only (kernel.cu:58, 78). */
int qcd_set_pair_layout(qcd_lattice* h, int on);
/* 1 if the FP32 store is in site pairs now, 0 if not (FP64: 0) */
int qcd_get_pair_layout(const qcd_lattice* h);
/* Fused pairs: streamed slices per CTA (0: automatic, enough CTAs for every
   SM several times over). */
int qcd_set_pair_tuning(qcd_lattice* h, int slices_per_cta);
/* Wavefront knobs (0 keeps the current value): sites per task (rounded up to
   a multiple of 256), passes chained per launch (1..4; more passes keep more
   slices live in L2) and fronts (a divisor of Lt leaving arcs of >= 2 slices:
   the ring is cut into that many arcs that advance together, multiplying the
   ready tasks and the live slices).  Defaults: 256 sites, as many passes as
   keep the live slices within ~64 MB, 1 front. */
int qcd_set_wave_tuning(qcd_lattice* h, int chunk_sites, int passes_per_launch, int fronts);
/* Autotuner.  Times per-phase launches, the fused pairs (FP32) and the
   wavefront (task sizes 256 / 512 / 1024 sites, 1..32 fronts whose live
   slices fit in L2, 1 or the largest chain of passes) for sweeps_per_trial
   sweeps each (0: 2) on this lattice (per-phase on the site-pair store where
   it applies, the others on float4 planes), then restores the lattice's
   links, their layout, streams and counters exactly and keeps the fastest
   schedule.  The choice is cached per (extents,
   precision, algorithm, boundary, n_or) for the life of the process, so later
   handles of the same shape reuse it without timing. */
typedef struct qcd_tuning {
  int schedule;           /* QCD_SCHED_PHASES, QCD_SCHED_WAVEFRONT or QCD_SCHED_PAIRS */
  int chunk_sites;        /* wavefront: sites per task; pairs: streamed slices per CTA (0 automatic) */
  int passes_per_launch, fronts;
  double ms_per_sweep;    /* measured time of the chosen candidate */
} qcd_tuning;
int qcd_autotune(qcd_lattice* h, int sweeps_per_trial, qcd_tuning* chosen);
/* Host-only planner of the wavefront (no GPU): for a program of n_phases
   phases (mu[n] in {0 y, 1 x, 2 t}, par[n] in {0, 1}) writes each phase's
   seam slice, start step and, in need[o*n_phases + n] (o = 0, 1, 2 for slice
   offsets -1, 0, +1), the latest earlier phase it waits for (-1: none). */
int qcd_wave_plan(const int* mu, const int* par, int n_phases, int* seam, int* start, int* need);
/* Self-test of the bounded waits: one wavefront pass in which the first task
   waits for a count no task produces; expected result QCD_ERR_TIMEOUT, with
   the CUDA context still usable (the links of that pass are left partly
   updated: re-initialise the lattice afterwards). */
int qcd_wave_selftest_timeout(qcd_lattice* h);

/* Random-generator checkpoint: qcd_rng_words(h) u32 words = the 6 x V/2
   words of the MRG32k3a streams (plane j of stream id at j * V/2 + id; the
   FP64 draws and every hot start) followed by the 64-bit drawing-phase
   counter and the 64-bit key of the FP32 sweep's counter-based draws (low
   words first).  No counterpart in the reference (a restart re-seeds with
   time(NULL), kernel.cu:79); with it a run resumed from a Config_ file
   continues the chain bit for bit. */
long long qcd_rng_words(const qcd_lattice* h);
int qcd_store_rng(qcd_lattice* h, uint32_t* host_out);
int qcd_load_rng(qcd_lattice* h, const uint32_t* host_in);

/* Philox4x32-10 block (Salmon et al., SC'11) on the host, the generator of
   the FP32 sweep: out = philox(ctr, key).  The heat-bath or Metropolis update
   of site id (sublattice index) in drawing phase k (6 per heat-bath or
   Metropolis pass, counted from the handle's creation) of a lattice with
   seed s reads blocks ctr = {id, b, k lo, k hi}, b = 0, 1, ..., key = {s lo,
   s hi}, word by word: float draws are ((w >> 8) + 1) / 2^24, double draws
   take two words.  Pure host code (no GPU). */
void qcd_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Lattice facts. */
long long qcd_volume(const qcd_lattice* h);
int qcd_get_params(const qcd_lattice* h, qcd_params* out);
/* Device pointer and byte size of the current link store (diagnostics,
   benchmarks).  Under QCD_SCHED_PAIRS each pass moves the links to the other
   of two stores, so the pointer holds until the next sweep.  An FP32 store
   is in site pairs when qcd_get_pair_layout says so. */
int qcd_link_store(const qcd_lattice* h, void** dev_ptr, size_t* bytes);

const char* qcd_last_error(const qcd_lattice* h);
const char* qcd_status_string(int status);

/* ------------------------------------------------------------------------
 * Batched replicas (no counterpart in the reference, which runs one lattice
 * per process).  Many independent lattices of different size, coupling,
 * boundary condition and start share one set of launches: a sweep of the
 * whole batch is the six phase launches of one lattice, each covering every
 * replica, and a measurement is one launch writing every replica's
 * (energy, plaquette).  qcd_batch_run captures one measurement interval as a
 * CUDA graph (per group of replicas, see qcd_batch_set_groups) and replays it.  Replica r starts (and, in FP64, draws) from
 * MRG32k3a streams curand_init(seed_r, stream_offset_r + id, 0); its FP32
 * sweep draws from the Philox counters of site stream_offset_r + id under key
 * seed_r.  With stream_offset 0 a replica reproduces a single lattice of the
 * same seed; giving replicas disjoint offset blocks under one seed keeps every
 * stream of the batch distinct.
 * ------------------------------------------------------------------------ */
typedef struct qcd_replica {
  int lt, lx, ly;          /* even extents */
  float beta;
  int boundary;            /* enum qcd_boundary */
  int hot;                 /* 1: hot start (rand_init2 / rand_init2_pcc), 0: cold */
  unsigned long long seed;
  long long stream_offset; /* first MRG32k3a subsequence / Philox site counter of this replica
                              (stream_offset + V/2 <= 2^40) */
} qcd_replica;
typedef struct qcd_batch qcd_batch;

/* common: algo, precision, epsilon, upd, n_or, renorm_every apply to every
   replica (its extents, beta, boundary and seed are ignored) */
int qcd_batch_create(const qcd_replica* replicas, int n, const qcd_params* common, qcd_batch** out);
int qcd_batch_destroy(qcd_batch* b);
int qcd_batch_set_stream(qcd_batch* b, void* stream);
/* seed every replica's streams and apply its start */
int qcd_batch_init(qcd_batch* b);
/* room for `capacity` measurements per replica (resets the series) */
int qcd_batch_reserve(qcd_batch* b, int capacity);
/* `sweeps` sweeps of every replica, measuring after every `measure_every`
   sweeps (0: never); with use_graph the interval runs as a CUDA graph */
int qcd_batch_run(qcd_batch* b, int sweeps, int measure_every, int use_graph);
/* Groups: the replicas are swept in groups of consecutive replicas holding
   at most bytes_per_group bytes of links (at least one replica each; 0: one
   group of everything; default 32 MB), each group going through all the
   sweeps of a qcd_batch_run while its links stay in L2 before the next group
   starts.  Replicas are independent and every group keeps its own
   drawing-phase counter and measurement cursor, so the results do not depend
   on the grouping. */
int qcd_batch_set_groups(qcd_batch* b, long long bytes_per_group);
/* number of groups */
int qcd_batch_groups(const qcd_batch* b);
/* Lanes (1..4, default 2): streams on which groups run at the same time,
   group g on lane g mod lanes, forked from and joined back into the batch's
   stream; one group's memory-bound measurement then overlaps another's
   phases. */
int qcd_batch_set_lanes(qcd_batch* b, int lanes);
/* Autotuner of the grouping: times sweeps_per_trial sweeps (0: 20; with a
   measurement after each when a series is reserved, as CUDA graphs) for one
   group of everything, the batch cut in halves on two lanes, and groups of
   128-16 MB of links on 1 to 4 lanes; restores the batch's
   links, streams, counters, cursors and series exactly, and keeps the fastest
   (its bytes per group, lanes and ms per sweep, where the pointers are not NULL). */
int qcd_batch_autotune(qcd_batch* b, int sweeps_per_trial, long long* bytes_out, int* lanes_out,
                       double* ms_per_sweep_out);
/* wait for the batch's stream; reports device-side errors */
int qcd_batch_synchronize(qcd_batch* b);
/* measurements taken so far (per replica) */
int qcd_batch_measured(qcd_batch* b);
int qcd_batch_series(qcd_batch* b, int replica, double* energy, double* plaquette, int n);
/* replica's configuration in the reference's AoS FP64 layout */
int qcd_batch_store_config(qcd_batch* b, int replica, double* aos_host);
long long qcd_batch_sites(const qcd_batch* b);
const char* qcd_batch_last_error(const qcd_batch* b);

/* ------------------------------------------------------------------------
 * Statistics of a measurement series (host only, no GPU).
 * The reference's naive mean / population variance and normalised
 * autocorrelation of lags 1..w (mean_variance, autocorrelation,
 * statistics.h:30-51), and what its README leaves to post-processing
 * (README.md:74): the binned error of the mean and the integrated
 * autocorrelation time tau_int = 1/2 + sum_{t<=W} rho(t) with the
 * Madras-Sokal window (smallest W >= c tau_int(W)) and its error.
 * ------------------------------------------------------------------------ */
int qcd_stats_mean_variance(const double* x, int n, double* mean, double* var);
int qcd_stats_autocorrelation(const double* x, int n, int w, double mean, double var, double* out);
int qcd_stats_binned(const double* x, int n, int bin, double* mean, double* err);
int qcd_stats_tau_int(const double* x, int n, double c, double* tau, int* window, double* dtau);

/* ------------------------------------------------------------------------
 * Random-number tape.  For stream id in [first, first+n_streams), seeded as
 * curand_init(seed, id, 0) exactly like setup_kernel (lattice_setup.h:15-21),
 * record the first n_draws draws.  Draw k is taken both as curand_uniform
 * and as curand_uniform_double from the same generator position, with the
 * CUDA float values the reference's heat-bath applies to one draw
 * (logf, cospif(2u), sincospif(2u); mc_updates.h:47-55).  `same_step` is 1
 * when both flavours advanced the generator identically.  Host-side replays
 * (the CPU oracle) consume this instead of re-implementing the generator.
 * ------------------------------------------------------------------------ */
typedef struct qcd_tape_record {
  double ud;
  float uf;
  float log_uf;
  float cospi_2uf;
  float sc_sin;
  float sc_cos;
  unsigned int same_step;
} qcd_tape_record;

int qcd_rng_tape(unsigned long long seed, long long first, int n_streams, int n_draws,
                 qcd_tape_record* host_out);

/* ------------------------------------------------------------------------
 * Measurement that allocates nothing.  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory when they measure: a
 * program that sized its lattice to fill the GPU, one whose device memory
 * belongs to the pooling allocator of its host framework, or a sweep loop
 * that cannot take the implicit device synchronisation of cudaMalloc /
 * cudaFree.  It needs no handle: it reads a configuration the caller holds
 * in device memory in the reference's AoS FP64 layout (V*12 doubles, the
 * layout of kernel.cu's `phid`, 16-byte aligned) and writes
 * out_dev[0] = energy, out_dev[1] = average plaquette (same definitions,
 * per-site arithmetic and summation order as qcd_measure) asynchronously on
 * `stream` (a cudaStream_t; NULL = the legacy default stream).  It calls no
 * cudaMalloc, cudaFree or other allocating routine: its reduction scratch is
 * a fixed array inside the library, present on every GPU that loads it until
 * the process exits.
 *
 * Limits: the scratch holds QCD_NOALLOC_MAX_BLOCKS partial sums (64 KB), which
 * is the most CTAs any measurement launches, whatever the lattice size: the
 * threads of a CTA stride over the sites.  The lattice itself is bounded only
 * by the 32-bit site indices, V/2 <= QCD_NOALLOC_MAX_HALF_SITES (the same bound
 * as qcd_create; 384^3 and larger fit); beyond it the call returns
 * QCD_ERR_UNSUPPORTED (and says so on stderr) without touching the device.
 * Every call looks up the scratch array's device address on the current
 * device (no allocation; with lazy module loading the first call on a device
 * also loads the library's kernels there): make that first call before any
 * stream capture.  All calls share the one scratch array: calls that can
 * overlap on the GPU (different streams, no ordering between them) race and
 * must not be issued.
 * ------------------------------------------------------------------------ */
#define QCD_NOALLOC_MAX_BLOCKS 4096
#define QCD_NOALLOC_MAX_HALF_SITES 357913940 /* the largest V/2 below 2^31 / 6 */
int qcd_measure_aos_noalloc(const double* phi_dev, int lt, int lx, int ly, int boundary,
                            double* out_dev, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* QCD2D_H */
