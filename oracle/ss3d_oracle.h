/*
 * ss3d_oracle.h -- CPU oracle for the SPECSIM3D spectral simulation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a literal C restatement of the reference
 * Fortran program (src/specsim3d.f90) used as the checker for the CUDA
 * implementation in specsim3d_b200/.  Only tests/, __graft_entry__.smoke() and
 * bench.py (CPU baseline leg and --impl reference) may load it.  The product
 * library never links, loads or calls anything in this directory.
 *
 * Parity status: pinned against the reference's own committed outputs of
 * seeded runs (docs/figures/scaling_cached.json RMS values at full double
 * precision; docs/figures/tables CSV files statistics at 4 digits), against the
 * Park-Miller known answer, and against the reference test scripts run as a
 * black box.  No Fortran compiler exists on the build or GPU machines, so the
 * Fortran binary itself was never run here.
 *
 * Array conventions follow the Fortran column-major layout: a grid array
 * a(nx,ny,nz) is stored with x fastest, index i + nx*(j + ny*k).
 * Complex arrays are interleaved (re, im) doubles.
 */
#ifndef SS3D_ORACLE_H
#define SS3D_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORA_MAXST 10

/* type(structure) f90:95-100 */
typedef struct {
    int itype;
    double sill, ahmax, ahmin, avert, az, dip, plg;
    double rot[3][3];   /* rot[r][c] = Fortran rot(r+1,c+1) */
    double axes[3][3];
} ora_struct;

/* setrot f90:107-139 */
void ora_setrot(ora_struct *s);
/* cutoff f90:142-150 */
double ora_cutoff(int itype);
/* covariance f90:153-178 */
double ora_covariance(const ora_struct *st, int nst, double nugget, double dx, double dy, double dz);
/* nextpow2 f90:181-188 */
int ora_nextpow2(int n);

/* Periodic grid sizing f90:1234-1253.  Returns 0, or 1 when the grid exceeds 2^27 nodes. */
int ora_periodic_grid(const ora_struct *st, int nst, const double d[3], const int n[3], int ipad, int np[3]);

/* Park-Miller stream f90:191-205 */
void ora_rng_seed(int iseed);           /* f90:1302-1303: seed + 10 discarded draws */
double ora_urand(void);
void ora_gauss_pair(double *g1, double *g2);
int64_t ora_rng_state(void);
void ora_rng_set_state(int64_t s);

/* FFT f90:208-304 (unscaled).  a is complex (interleaved) a(nx,ny,nz). */
void ora_fft1d(double *x, int n, const double *tw);
void ora_twiddles(int n, int isign, double *tw);
void ora_fft3d(double *a, int nx, int ny, int nz, int isign);

/* Spectrum statistics printed at f90:1289-1292 */
typedef struct {
    double c0, maximag, maxreal, spos, sneg;
} ora_spec_stats;

/* Covariance grid + forward FFT + /N + clip/sqrt, f90:1256-1292.
 * amp: real array (npx,npy,npz).  Returns 0 on success. */
int ora_spectrum(const ora_struct *st, int nst, double nugget, const double d[3], const int np[3],
                 double *amp, ora_spec_stats *stats);

/* Hermitian coefficient fill for ONE realization from the current RNG state,
 * f90:1306-1334.  c: complex (npx,npy,npz), overwritten at every index. */
void ora_fill_coefficients(const double *amp, const int np[3], int igauss, double *c);

/* Like ora_fill_coefficients but records, for every index, the RNG state right
 * after the first draw that produced it (0 where no draw was made, i.e. the
 * conjugate partner of an earlier index).  Used to pin the jump-ahead stream. */
void ora_fill_states(const int np[3], int igauss, int64_t *first_state);

/* Realizations f90:1302-1345: seeds the stream, fills, inverse FFT, crops.
 * res: (nx,ny,nz,nreal) doubles.  zstats (may be NULL): 3 doubles per realization
 * (mean, variance, max|Im|). */
int ora_realize(const double *amp, const int np[3], const int n[3], int iseed, int nreal, int igauss,
                double *res, double *zstats);
/* the same for realizations r_first+1 .. r_first+nreal of the serial run */
int ora_realize_range(const double *amp, const int np[3], const int n[3], int iseed, int r_first, int nreal,
                      int igauss, double *res, double *zstats);

/* Experimental variogram, f90:394-431 */
int64_t ora_npair_count(int nx, int ny, int nz, int lx, int ly, int lz);
double ora_vario_lag(const double *f, int nx, int ny, int nz, int lx, int ly, int lz);
/* gam(nlagmax, ndir, nreal) for all (dir, lag, realization), f90:462-480 */
void ora_vario_all(const double *res, const int n[3], int nreal, int ndir, const int *sx, const int *sy,
                   const int *sz, const int *nlag, double *gam);

/* GSLIB helpers, f90:557-697 */
double ora_gcum(double x);
double ora_gauinv(double p);
void ora_heapsort_idx(const double *key, int *idx, int n);   /* idx is 1-based values */
void ora_nscore(int nd, const double *v, const double *w, double *g, int *nt, double *vr, double *gt);
double ora_backtr(double y, int nt, const double *vr, const double *gt, double zmin, double zmax,
                  int lt, double ltp, int ut, double utp);

/* Conditioning parameters, f90:740-750 */
typedef struct {
    int ixc, iyc, izc, ivc, iwc, itrans, ltail, utail, ndmax;
    double tmin, tmax, skmean, zlo, zhi, ltpar, utpar, rmax, rmed, rvert, sa1, sa2, sa3;
} ora_cond_params;

typedef struct {
    int nd, nmerged, nout, nsb[3];
    int64_t nsum;
    int nfail, nnone, nexact;
} ora_cond_stats;

/* Conditioning of res in place on the given (already read) data rows,
 * f90:782-924.  raw_rows: nrows x nvar values (row-major).  Writes the nscore
 * table (vrt, gtt, length nd) and the data used (dxs,dys,dzs,dval,dg) when the
 * out pointers are non-NULL (each must hold nrows values).  Returns 0, or a
 * nonzero code when no datum falls inside the grid. */
int ora_condition(double *res, const int n[3], int nreal, const double xmin[3], const double d[3],
                  const ora_struct *st, int nst, double nugget, const ora_cond_params *cp,
                  const double *raw_rows, int nrows, int nvar, ora_cond_stats *cs,
                  double *vrt, double *gtt, double *dxs, double *dys, double *dzs, double *dval, double *dg);

/* Command-line driver (the full program, f90:1085-1418). */
int ora_main(int argc, char **argv);

#ifdef __cplusplus
}
#endif
#endif
