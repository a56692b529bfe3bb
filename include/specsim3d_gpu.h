/*
 * specsim3d_gpu.h -- C ABI of the B200 implementation of the SPECSIM3D
 * spectral simulation path (library: specsim3d_b200/lib/libspecsim3d_gpu.so).
 *
 * The reference (src/specsim3d.f90) has no library interface: its stages are
 * inline code of `program specsim3d`.  Every entry point below names the
 * reference lines whose behaviour it replaces.  Plain C types only; no
 * CUDA or torch types appear in the signatures.
 *
 * Conventions
 *   - Every function returns an int status: 0 on success, a SS3D_E* code on
 *     failure, with a message available from ss3d_last_error().  The library
 *     never calls exit().
 *   - Fortran integer -> int32_t (int), real(dp) -> double, integer(8) -> int64_t.
 *   - Grid arrays follow the Fortran layout res(nx,ny,nz,nreal): x fastest, i.e.
 *     C order [nreal][nz][ny][nx].
 *   - Output and in/out arrays may be host or device pointers; the library
 *     detects which.  The library owns device memory behind opaque handles.
 *   - A spectrum handle is read-only after creation: several host threads may
 *     call ss3d_realize on it at once, each on its own stream (set per thread
 *     with ss3d_set_stream; default: the legacy default stream).  Every call
 *     returns after its results are complete.
 */
#ifndef SPECSIM3D_GPU_H
#define SPECSIM3D_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SS3D_OK 0
#define SS3D_EINVAL 1     /* invalid argument (message says which) */
#define SS3D_ECUDA 2      /* CUDA runtime error */
#define SS3D_ENOMEM 3     /* device memory exhausted */
#define SS3D_ETOOLARGE 4  /* periodic grid above 2^27 nodes (f90:1253) or axis above the supported length */
#define SS3D_ENODATA 5    /* conditioning: no datum inside the grid (f90:804) */

#define SS3D_FP64 0       /* plain form: FP64 throughout */
#define SS3D_FP32 1       /* precision form: FP32 synthesis and FFTs on the FP64 spectrum */

#define SS3D_OUT_F32 0    /* float32 output (the .bin/.vtk/.vti value type) */
#define SS3D_OUT_F64 1    /* float64 output (the reference's res array) */

/* One nested structure: `itype sill ahmax ahmin avert azimuth dip plunge`
 * (type(structure), f90:95-100; parameter-file line f90:1167-1168). */
typedef struct ss3d_struct {
    int itype;          /* 1 spherical, 2 exponential, 3 gaussian */
    double sill, ahmax, ahmin, avert, azimuth, dip, plunge;
} ss3d_struct;

/* Spectrum diagnostics printed by the reference at f90:1289-1292. */
typedef struct ss3d_spec_stats {
    int np[3];          /* periodic grid npx, npy, npz (f90:1234-1251) */
    double c0;          /* C(0), "target variance" */
    double maximag;     /* max |Im S| */
    double maxreal;     /* max |Re S| */
    double spos;        /* sum of positive S */
    double sneg;        /* sum of negative S (clipped to zero in amp) */
} ss3d_spec_stats;

typedef struct ss3d_spectrum ss3d_spectrum;

/* ---------------------------------------------------------------- host-side model */

/* GSLIB rotation of one structure: rot and axes are 3x3 row-major
 * (rot[3*r+c] = Fortran rot(r+1,c+1)).  Replaces setrot, f90:107-139. */
int ss3d_setrot(const ss3d_struct *s, double rot[9], double axes[9]);

/* Covariance C(h) of nst nested structures plus nugget at lag (dx,dy,dz).
 * Replaces covariance, f90:153-178. */
int ss3d_covariance(const ss3d_struct *st, int nst, double nugget, double dx, double dy, double dz, double *c);

/* Periodic grid of the ipad rule.  Replaces nextpow2/cutoff and the grid block
 * f90:142-188, f90:1234-1253; returns SS3D_ETOOLARGE above 2^27 nodes. */
int ss3d_grid_size(const ss3d_struct *st, int nst, const double d[3], const int n[3], int ipad, int np[3]);

/* ---------------------------------------------------------------- spectrum */

/* Covariance grid on the periodic grid, forward 3D FFT, S = FFT/N and
 * amp = sqrt(max(Re S, 0)), all on the GPU in FP64, kept resident in device
 * memory.  Replaces f90:1256-1292.  stats may be NULL. */
int ss3d_spectrum_create(const ss3d_struct *st, int nst, double nugget, const double d[3], const int n[3], int ipad,
                         ss3d_spectrum **out, ss3d_spec_stats *stats);
void ss3d_spectrum_free(ss3d_spectrum *sp);

/* Grid sizes and stats of a spectrum (np, n may be NULL). */
int ss3d_spectrum_info(const ss3d_spectrum *sp, int np[3], int n[3], ss3d_spec_stats *stats);

/* Device memory held by the spectrum (bytes), for admission control. */
int64_t ss3d_spectrum_bytes(const ss3d_spectrum *sp);

/* Copy of the FP64 amplitude on the Hermitian half spectrum, amp[k][j][i],
 * i < npx/2+1 (host pointer).  Test hook for the f90:1277-1288 values. */
int ss3d_spectrum_amp(const ss3d_spectrum *sp, double *amp);

/* ---------------------------------------------------------------- realizations */

/* Realizations r_first .. r_first+nreal-1 (0-based) of the reference stream for
 * seed iseed: Hermitian coefficient synthesis with the Park-Miller stream
 * reproduced bit-exactly by jump-ahead, inverse 3D FFT, crop to nx,ny,nz.
 * Replaces f90:1302-1345.  r_first = 0, nreal = N gives exactly the
 * reference's realizations 1..N; any sub-range gives the same values as the
 * corresponding part of the full run (exact sharding).
 *   igauss     0 fixed amplitudes + random phases, 1 Gaussian coefficients
 *   precision  SS3D_FP64 or SS3D_FP32
 *   out        res(nx,ny,nz,nreal) of out_dtype (SS3D_OUT_F32 / SS3D_OUT_F64),
 *              host or device memory
 *   zstats     NULL or 3*nreal doubles: mean, variance, max|Im| per realization
 *              (the line printed at f90:1343-1344; max|Im| is 0 because the
 *              Hermitian half-spectrum inverse is real by construction). */
/*   A device out must belong to the spectrum's device and, when nx is even,
 *   start on a multiple of twice the element size (rows are stored as pairs);
 *   otherwise SS3D_EINVAL before any work.  Host out has no alignment rule. */
int ss3d_realize(const ss3d_spectrum *sp, int iseed, int64_t r_first, int nreal, int igauss, int precision,
                 void *out, int out_dtype, double *zstats);

/* State of the reference's Park-Miller stream right after the first draw of
 * row (j, k) (0-based) of realization r (0-based) on the periodic grid np, as
 * the realization kernels compute it by jump-ahead (host only, no GPU).  The
 * reference draws this stream serially (f90:1302-1334); the function lets a
 * host plan and check a split of realizations over processes or GPUs. */
int ss3d_row_state(const int np[3], int igauss, int iseed, int64_t r, int j, int k, uint32_t *state);

/* Test hooks for the synthesis (host output arrays, half spectrum [k][j][i],
 * i < npx/2+1):
 *   ss3d_debug_states: Park-Miller state after the first draw that produced
 *     each coefficient of realization r (the partner's draw for conjugate rows)
 *   ss3d_debug_coefficients: the coefficients themselves (re, im interleaved). */
int ss3d_debug_states(const ss3d_spectrum *sp, int iseed, int64_t r, int igauss, uint32_t *states);
int ss3d_debug_coefficients(const ss3d_spectrum *sp, int iseed, int64_t r, int igauss, int precision, double *coef);

/* Unscaled 3D FFT of a full complex grid a(nx,ny,nz) in place, FP64, x fastest,
 * interleaved (re, im) doubles, host or device memory: isign -1 forward
 * (e^{-2 pi i k n/N}), +1 inverse.  Replaces fft3d, f90:254-304 (exported for
 * unit tests; the simulation path itself uses Hermitian half-spectrum passes).
 * Every axis a power of two up to 2048, at most 2^27 nodes. */
int ss3d_fft3d(double *a, int nx, int ny, int nz, int isign);

/* Realizations like ss3d_realize, but without allocating device memory.  No
 * counterpart in the reference (the Fortran program allocates its own arrays).
 * For callers that cannot call cudaMalloc when they need realizations: an
 * application that has handed the GPU's memory to its own pool (a serving
 * process that reserves HBM up front), or a latency-bound loop that cannot
 * afford the device-wide synchronisation of cudaMalloc/cudaFree.  All scratch
 * lives in one fixed array of SS3D_NOALLOC_SCRATCH_BYTES that every GPU loading
 * the library holds until exit.  A call needs about nz * npy * (npx/2 + 2) * 8
 * bytes (FP32; 16 for FP64; nz is replaced by 1 when npz = 1) plus 0.5 MB of
 * tables: a 128^3 grid on its 256^3 periodic grid fits in FP32 (34 MB) but is
 * refused in FP64 (68 MB); the 256^3 grid on 512^3 is refused in both.  Refused
 * grids return SS3D_ETOOLARGE and a message giving the bytes needed.  out must
 * be device memory of the spectrum's device, which must be the current device
 * (SS3D_EINVAL otherwise, before any work).  The first call on a device copies
 * the constant tables into the array and synchronises the device: make that
 * first call before any stream capture begins.  Every call shares and
 * overwrites the one array, so calls that overlap on the GPU race. */
#define SS3D_NOALLOC_SCRATCH_BYTES (64u << 20)
int ss3d_realize_noalloc(const ss3d_spectrum *sp, int iseed, int64_t r_first, int nreal, int igauss, int precision,
                         void *out, int out_dtype);

/* Autotuner of the realization kernels (no counterpart in the reference, whose
 * FFT has a single code path).  For the grid of sp, times each compiled tile
 * variant of the synthesis pass, the middle column pass and the C2R row pass
 * on nreal realizations and keeps the fastest for later calls in this process
 * (per precision and transform length).  chosen (may be NULL) receives the
 * variants picked for {middle pass, synthesis pass, row pass}. */
int ss3d_autotune(const ss3d_spectrum *sp, int igauss, int precision, int nreal, int chosen[3]);

/* Loads every kernel of the library on the current device now.  CUDA loads a
 * kernel when it is first launched by default, and loading one may
 * synchronise the device: a process that runs other work beside the library
 * (a server, several threads) can take the loads up front.  ss3d_server_create
 * calls it.  No counterpart in the reference. */
int ss3d_preload_kernels(void);

/* Explicit variant of kernel kind 0 middle pass, 1 synthesis pass, 2 row
 * pass, for one precision and transform length 2^logn: 0..3 one line per
 * thread; for the FP32 column passes (kinds 0, 1) also 4..7, two adjacent
 * lines per thread on the packed FP32 instructions; for the FP32 middle pass
 * also 8 and 9, tiles brought into shared memory by bulk tensor copies (one
 * and two lines per thread); for the row pass also 4, each row held in the
 * registers of one warp (row lengths 8..512 in FP32, 8..256 in FP64; other
 * lengths run variant 0), and in FP32 5, the middle and row passes of a plane
 * in one thread-block cluster (3-D grids, float output without statistics,
 * y lengths 64..512, row lengths 128..512; elsewhere variant 4), and 6, two
 * rows per lane on the packed FP32 instructions (row lengths 8..256;
 * elsewhere variant 4).  Every variant computes the same values; they differ
 * in tile shape and instruction form only. */
int ss3d_set_variant(int kind, int precision, int logn, int variant);

/* ---------------------------------------------------------------- batched form */

/* Many realizations of many grids in one CUDA-graph launch (FP32 synthesis and
 * transforms, float output).  A job asks for realizations r_first ..
 * r_first+nreal-1 of one spectrum into a DEVICE array out[nreal][nz][ny][nx];
 * each result equals ss3d_realize(sp, iseed, r_first, nreal, igauss,
 * SS3D_FP32, out, SS3D_OUT_F32, NULL) bit for bit.  The batch owns its work
 * space (the complex grids of every job) and replays one graph on each run;
 * the spectra and output arrays must outlive it.  The reference simulates one
 * grid per process (its realization loop, f90:1300-1345); this form has no
 * counterpart there. */
typedef struct ss3d_batch ss3d_batch;
typedef struct ss3d_batch_job {
    const ss3d_spectrum *sp;
    int iseed;
    int igauss;
    int64_t r_first;
    int nreal;
    float *out;
} ss3d_batch_job;

int ss3d_batch_create(const ss3d_batch_job *jobs, int njobs, ss3d_batch **out);
/* One graph launch on the calling thread's stream; returns when done. */
int ss3d_batch_run(ss3d_batch *b);
/* Times the schedules and tile variants, keeps the fastest and re-captures the
 * graph; results do not change. */
int ss3d_batch_autotune(ss3d_batch *b);
/* Output cells of one run, kernel launches of one run, and for the persistent
 * schedule its CTAs and work items per pass (all outputs may be NULL). */
int ss3d_batch_info(const ss3d_batch *b, int64_t *cells, int grid[3], int items[3], int *kernels);
/* One run timed with CUDA events outside the graph: ms[0..2] the synthesis,
 * middle and row passes (persistent schedule; -1 for chains), ms[3] the run. */
int ss3d_batch_time(ss3d_batch *b, float ms[4]);
/* Schedule: sched 0 chains (one chain of per-call kernels per job on parallel
 * graph branches), 1 persistent (three kernels over one work list of every
 * job's tiles; needs periodic axes of 16..1024 nodes and npx >= 16).  For the
 * persistent schedule per pass: tile variant etv (0: 16, 1: 8 elements per
 * thread), mode (0 strided items, 1 contiguous items, 2 one CTA per item) and
 * CTAs per SM (0: occupancy limit). */
int ss3d_batch_schedule(const ss3d_batch *b, int *sched, int etv[3], int mode[3], int cps[3]);
int ss3d_batch_set_schedule(ss3d_batch *b, int sched, int pass, int etv, int mode, int cps);
/* Chains schedule: each job's realizations run as `split` consecutive
 * sub-chains on separate branches, sub-chain q starting when the synthesis of
 * sub-chain q-1 has ended, so that syntheses overlap the middle and row passes
 * of earlier sub-chains (1: one chain per job; chosen by ss3d_batch_autotune).
 * Results do not depend on it. */
int ss3d_batch_split(const ss3d_batch *b, int *split);
int ss3d_batch_set_split(ss3d_batch *b, int split);
void ss3d_batch_free(ss3d_batch *b);

/* ---------------------------------------------------------------- variogram */

/* Experimental semivariograms of nreal fields res(nx,ny,nz,nreal) (FP64, host or
 * device) along ndir integer directions (sx,sy,sz), lags 1..nlag[d], over all
 * node pairs.  gam(nlagmax, ndir, nreal) column-major as in the reference;
 * npairs(nlagmax, ndir) (may be NULL) are the exact pair counts.
 * Replaces npair_count / vario_lag / the task loop of vario_report, f90:394-480. */
int ss3d_vario(const double *res, const int n[3], int nreal, int ndir, const int *sx, const int *sy, const int *sz,
               const int *nlag, double *gam, int64_t *npairs);

/* ---------------------------------------------------------------- conditioning */

/* Conditioning block of the parameter file (f90:740-750). */
typedef struct ss3d_cond_params {
    int ixc, iyc, izc, ivc, iwc;   /* data columns (1-based; izc, iwc may be 0) */
    double tmin, tmax;             /* trimming limits */
    int itrans;                    /* 1: normal score + back transform */
    double skmean;                 /* mean removed when itrans = 0 */
    double zmin, zmax;             /* back-transform limits */
    int ltail; double ltpar;       /* lower tail (1 linear, 2 power) */
    int utail; double utpar;       /* upper tail (1 linear, 2 power, 4 hyperbolic) */
    double radius[3];              /* search radii: max, med, vert */
    double angles[3];              /* search angles: azimuth, dip, plunge */
    int ndmax;                     /* 1..100 */
} ss3d_cond_params;

typedef struct ss3d_cond_stats {
    int nd, nmerged, nout;         /* data used, merged, outside the grid */
    int nsb[3];                    /* super blocks per axis */
    int64_t nsum;                  /* total neighbours over all nodes */
    int nfail, nnone, nexact;      /* regularised systems, empty nodes, data nodes */
    double data_mean, data_var;    /* of the normal scores (itrans = 1) */
} ss3d_cond_stats;

/* Conditioning by kriging of the residual: data snapping and merging, optional
 * normal-score transform (host), super-block neighbour search and simple
 * kriging at every node (GPU), back transform (GPU).  res(nx,ny,nz,nreal) FP64
 * host or device, modified in place.  rows: nrows x nvar data values
 * (row-major, the numeric rows of the GSLIB data file).  precision SS3D_FP64
 * solves in FP64; SS3D_FP32 solves in FP32 with one FP64 residual refinement.
 * The optional outputs (each of nrows doubles, may be NULL) receive the
 * normal-score table (vrt, gtt) and the data actually used.
 * Replaces condition_field f90:782-924, krige_node f90:949-1038,
 * chol_solve f90:1040-1079, nscore/backtr f90:557-697. */
int ss3d_condition(double *res, const int n[3], int nreal, const double xmin[3], const double d[3],
                   const ss3d_struct *st, int nst, double nugget, const ss3d_cond_params *cp, const double *rows,
                   int nrows, int nvar, int precision, ss3d_cond_stats *cs, double *vrt, double *gtt, double *dxs,
                   double *dys, double *dzs, double *dval, double *dg);

/* ---------------------------------------------------------------- serving form */

/* A request loop over the simulation path (no counterpart in the reference,
 * which runs one parameter file per process).  ss3d_server_submit queues a
 * request and returns at once; `slots` worker threads, each with its own CUDA
 * stream and work space, admit queued requests in arrival order as soon as a
 * slot is free and the request's device footprint (work space, conditioning
 * temporaries, and the spectrum with its build temporaries when the model is
 * not resident) fits the HBM budget (freed memory that the library's
 * stream-ordered pool keeps mapped is not counted); a request that does not
 * fit waits, and
 * later requests may pass it at most max_bypass times.  Spectra stay resident
 * in an LRU cache keyed by model, grid and ipad.  Each request runs
 * ss3d_spectrum_create (on a cache miss), ss3d_realize and, with data,
 * ss3d_condition, so its result equals the same calls made alone.
 * The caller keeps `out` and `rows` alive until ss3d_server_wait returns. */
typedef struct ss3d_server ss3d_server;

typedef struct ss3d_server_config {
    int slots;                   /* requests on the GPU at once (1..64) */
    int max_bypass;              /* passes of a waiting queue head (0: 16) */
    int max_cond;                /* conditional requests on the GPU at once (0: 2); they run
                                    on low-priority streams, the others on high-priority ones */
    int64_t hbm_budget;          /* device bytes for spectra and work (0: 80 % of free memory) */
    int64_t cache_budget;        /* bytes of idle spectra kept (0: half the budget) */
    int64_t retain_bytes;        /* largest work space a slot keeps between requests
                                    (0: min(4 GiB, hbm_budget / (2 slots))); kept bytes
                                    stay charged to the budget, and an idle slot gives
                                    them back when the queue head does not fit */
    double dry_run_ns_per_cell;  /* > 0: no GPU work, sleeps of this many ns per cell
                                    (scheduler tests); needs an explicit hbm_budget */
    int64_t premap_bytes;        /* device bytes mapped into the stream-ordered pool at
                                    creation (best effort, at most the budget; 0: none):
                                    mapping pages while requests run stalls the device
                                    for all of them */
} ss3d_server_config;

typedef struct ss3d_request {
    const ss3d_struct *st;       /* model: nst structures and the nugget */
    int nst;
    double nugget;
    double d[3];                 /* cell size */
    int n[3];                    /* grid */
    int ipad;
    int iseed, igauss;
    int64_t r_first;
    int nreal;
    int precision;               /* SS3D_FP64 or SS3D_FP32 */
    void *out;                   /* res(nx,ny,nz,nreal), host or device */
    int out_dtype;               /* SS3D_OUT_F32 / SS3D_OUT_F64 (F64 with conditioning data) */
    double t_arrival;            /* arrival on the server clock (< 0: the submit time) */
    /* conditioning (nrows = 0: unconditional), as ss3d_condition */
    const ss3d_cond_params *cp;
    const double *rows;
    int nrows, nvar;
    double xmin[3];
} ss3d_request;

typedef struct ss3d_result {
    int status;                  /* SS3D_OK or the failing stage's code */
    int cache_hit;               /* the spectrum was resident or being built */
    double t_arrival, t_submit, t_admit, t_done;   /* seconds on the server clock */
    int64_t footprint;           /* device bytes the request was admitted with */
} ss3d_result;

typedef struct ss3d_serve_stats {
    int64_t submitted, completed, failed;
    int64_t cache_hits, cache_misses, evictions;
    int64_t cells;               /* output cells of completed requests */
    int64_t peak_bytes;          /* peak of charged + cached bytes */
    int64_t peak_running, running, queued, cached_spectra;
    int64_t cache_bytes, charged_bytes, budget_bytes;
} ss3d_serve_stats;

int ss3d_server_create(const ss3d_server_config *cfg, ss3d_server **out);
int ss3d_server_submit(ss3d_server *s, const ss3d_request *req, int64_t *ticket);
/* Blocks until the request is done; returns its status (message in
 * ss3d_last_error on this thread).  Each ticket is waited for once. */
int ss3d_server_wait(ss3d_server *s, int64_t ticket, ss3d_result *res);
int ss3d_server_stats(ss3d_server *s, ss3d_serve_stats *stats);
double ss3d_server_clock(ss3d_server *s);   /* seconds since creation */
/* Stops the slots after the running requests; queued requests fail. */
void ss3d_server_free(ss3d_server *s);

/* ---------------------------------------------------------------- runtime */

/* Stream (a cudaStream_t passed as void*) on which later calls from the
 * calling host thread issue work; NULL selects the legacy default stream. */
int ss3d_set_stream(void *stream);

/* The realization work space is kept per host thread and device and grows on
 * demand.  ss3d_realize_workspace_bytes gives the device bytes a call of nreal
 * realizations needs (host_out: 1 for a host output array), for admission
 * control; -1 on invalid arguments.  ss3d_release_workspace frees the calling
 * thread's work space. */
int64_t ss3d_realize_workspace_bytes(const ss3d_spectrum *sp, int nreal, int precision, int host_out);
int ss3d_release_workspace(void);

/* The library takes its device memory from the device's stream-ordered pool
 * and keeps freed memory mapped for its next calls; ss3d_trim_pool synchronises
 * the device and returns the pool's unused memory to it. */
int ss3d_trim_pool(void);

/* Message of the last failing call on this thread ("" if none). */
const char *ss3d_last_error(void);

/* Library version string. */
const char *ss3d_version(void);

/* Stage timing of the realization path (the reference prints only wall-clock
 * totals, f90:1299-1300, 1350-1351).  With profiling on, ss3d_realize records
 * CUDA events around each stage on its stream; ss3d_profile_read returns the
 * accumulated milliseconds and launch counts per stage since the last reset:
 *   0 row states, 1 synthesis + first inverse pass, 2 middle inverse pass,
 *   3 C2R x pass + crop, 4 statistics.
 * launches_total counts every kernel launched by the library. */
#define SS3D_NSTAGE 5
int ss3d_profile(int enable);
int ss3d_profile_read(double ms[SS3D_NSTAGE], int64_t launches[SS3D_NSTAGE], int64_t *launches_total);

#ifdef __cplusplus
}
#endif
#endif
