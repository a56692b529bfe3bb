/*
 * ss3d_oracle.c -- CPU oracle: literal C restatement of the numerical core of
 * the reference program src/specsim3d.f90 (SPECSIM3D).
 *
 * TEST INFRASTRUCTURE ONLY (see ss3d_oracle.h).  Each function cites the
 * Fortran lines it restates.  Expression order follows the Fortran source and
 * the file is compiled with -ffp-contract=off (no FMA contraction), as
 * gfortran -O3 on x86-64 without -march=native produces no FMA either.
 * Serial loops of the reference (the coefficient fill, the crop) stay serial;
 * loops that the reference runs under OpenMP are independent per iteration, so
 * their results do not depend on the thread count.
 */
#include "ss3d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double PI = 3.14159265358979323846; /* f90:92 */

/* ------------------------------------------------------------------ model */

/* setrot, f90:107-139 */
void ora_setrot(ora_struct *s)
{
    double deg = PI / 180.0;
    double alpha;
    if (s->az >= 0.0 && s->az < 270.0)
        alpha = (90.0 - s->az) * deg;
    else
        alpha = (450.0 - s->az) * deg;
    double beta = -(s->dip * deg);
    double theta = s->plg * deg;
    double sina = sin(alpha), cosa = cos(alpha);
    double sinb = sin(beta), cosb = cos(beta);
    double sint = sin(theta), cost = cos(theta);
    double anis1 = s->ahmin / s->ahmax;
    double anis2 = s->avert / s->ahmax;
    double afac1 = 1.0 / fmax(anis1, 1.0e-20);
    double afac2 = 1.0 / fmax(anis2, 1.0e-20);
    s->rot[0][0] = cosb * cosa;
    s->rot[0][1] = cosb * sina;
    s->rot[0][2] = -sinb;
    s->rot[1][0] = afac1 * (-(cost * sina) + sint * sinb * cosa);
    s->rot[1][1] = afac1 * (cost * cosa + sint * sinb * sina);
    s->rot[1][2] = afac1 * (sint * cosb);
    s->rot[2][0] = afac2 * (sint * sina + cost * sinb * cosa);
    s->rot[2][1] = afac2 * (-(sint * cosa) + cost * sinb * sina);
    s->rot[2][2] = afac2 * (cost * cosb);
    for (int c = 0; c < 3; c++) {
        s->axes[0][c] = s->rot[0][c] * s->ahmax;
        s->axes[1][c] = s->rot[1][c] / afac1 * s->ahmin;
        s->axes[2][c] = s->rot[2][c] / afac2 * s->avert;
    }
}

/* cutoff, f90:142-150 */
double ora_cutoff(int itype)
{
    if (itype == 1) return 1.0;
    if (itype == 2) return 2.3;
    return 1.6;
}

/* covariance, f90:153-178 */
double ora_covariance(const ora_struct *st, int nst, double nugget, double dx, double dy, double dz)
{
    double c = 0.0;
    if (dx == 0.0 && dy == 0.0 && dz == 0.0) c = nugget;
    for (int i = 0; i < nst; i++) {
        const ora_struct *s = &st[i];
        double rx = s->rot[0][0] * dx + s->rot[0][1] * dy + s->rot[0][2] * dz;
        double ry = s->rot[1][0] * dx + s->rot[1][1] * dy + s->rot[1][2] * dz;
        double rz = s->rot[2][0] * dx + s->rot[2][1] * dy + s->rot[2][2] * dz;
        double h = sqrt(rx * rx + ry * ry + rz * rz);
        double hr = h / s->ahmax;
        if (s->itype == 1) {
            if (hr < 1.0) c = c + s->sill * (1.0 - 1.5 * hr + 0.5 * (hr * hr * hr));
        } else if (s->itype == 2) {
            c = c + s->sill * exp(-3.0 * hr);
        } else {
            c = c + s->sill * exp(-(3.0 * hr * hr));
        }
    }
    return c;
}

/* nextpow2, f90:181-188 */
int ora_nextpow2(int n)
{
    int m = 1;
    while (m < n) m = m * 2;
    return m;
}

/* periodic grid size, f90:1234-1253 */
int ora_periodic_grid(const ora_struct *st, int nst, const double d[3], const int n[3], int ipad, int np[3])
{
    np[0] = ora_nextpow2(n[0]);
    np[1] = ora_nextpow2(n[1]);
    np[2] = ora_nextpow2(n[2]);
    if (ipad == 1) {
        double e[3] = {0.0, 0.0, 0.0};
        for (int s = 0; s < nst; s++) {
            for (int a = 0; a < 3; a++) {
                double ss = st[s].axes[0][a] * st[s].axes[0][a];
                ss = ss + st[s].axes[1][a] * st[s].axes[1][a];
                ss = ss + st[s].axes[2][a] * st[s].axes[2][a];
                double v = ora_cutoff(st[s].itype) * sqrt(ss) / d[a];
                e[a] = fmax(e[a], v);
            }
        }
        int r[3];
        for (int a = 0; a < 3; a++) r[a] = (int)ceil(e[a]);
        np[0] = ora_nextpow2(n[0] + r[0] > 2 * r[0] ? n[0] + r[0] : 2 * r[0]);
        np[1] = ora_nextpow2(n[1] + r[1] > 2 * r[1] ? n[1] + r[1] : 2 * r[1]);
        if (n[2] > 1)
            np[2] = ora_nextpow2(n[2] + r[2] > 2 * r[2] ? n[2] + r[2] : 2 * r[2]);
        else
            np[2] = 1;
    }
    double ntot = (double)np[0] * (double)np[1] * (double)np[2];
    return ntot > 134217728.0 ? 1 : 0;
}

/* ------------------------------------------------------------------ RNG */

static int64_t rng_state = 1; /* f90:102 */

/* urand, f90:191-195 */
double ora_urand(void)
{
    rng_state = (16807LL * rng_state) % 2147483647LL;
    return (double)rng_state / 2147483647.0;
}

/* gauss_pair, f90:198-205 */
void ora_gauss_pair(double *g1, double *g2)
{
    double u1 = ora_urand();
    double u2 = ora_urand();
    double rr = sqrt(-2.0 * log(u1));
    *g1 = rr * cos(2.0 * PI * u2);
    *g2 = rr * sin(2.0 * PI * u2);
}

/* seeding, f90:1302-1303 */
void ora_rng_seed(int iseed)
{
    int64_t a = iseed < 0 ? -(int64_t)iseed : (int64_t)iseed;
    rng_state = a % 2147483646LL + 1;
    for (int i = 0; i < 10; i++) (void)ora_urand();
}

int64_t ora_rng_state(void) { return rng_state; }
void ora_rng_set_state(int64_t s) { rng_state = s; }

/* ------------------------------------------------------------------ FFT */

/* complex product in the order of gfortran's expansion: (ac - bd, ad + bc) */
static inline void cmul(double ar, double ai, double br, double bi, double *re, double *im)
{
    *re = ar * br - ai * bi;
    *im = ar * bi + ai * br;
}

/* fft1d, f90:208-241: iterative radix-2 DIT with bit reversal (1-based indices) */
void ora_fft1d(double *x, int n, const double *tw)
{
    if (n < 2) return;
    int j = 1;
    for (int i = 1; i <= n - 1; i++) {
        if (i < j) {
            double tr = x[2 * (i - 1)], ti = x[2 * (i - 1) + 1];
            x[2 * (i - 1)] = x[2 * (j - 1)];
            x[2 * (i - 1) + 1] = x[2 * (j - 1) + 1];
            x[2 * (j - 1)] = tr;
            x[2 * (j - 1) + 1] = ti;
        }
        int m = n / 2;
        while (m >= 1 && j > m) {
            j = j - m;
            m = m / 2;
        }
        j = j + m;
    }
    for (int len = 2; len <= n; len *= 2) {
        int half = len / 2, step = n / len;
        for (int i = 1; i <= n; i += len) {
            for (int k = 0; k <= half - 1; k++) {
                double *pu = &x[2 * (i + k - 1)];
                double *pv = &x[2 * (i + k + half - 1)];
                double ur = pu[0], ui = pu[1];
                double tr, ti;
                cmul(tw[2 * (k * step)], tw[2 * (k * step) + 1], pv[0], pv[1], &tr, &ti);
                pu[0] = ur + tr;
                pu[1] = ui + ti;
                pv[0] = ur - tr;
                pv[1] = ui - ti;
            }
        }
    }
}

/* twiddles, f90:244-251: tw(k+1) = cos(2 pi k/n) + i isign sin(2 pi k/n) */
void ora_twiddles(int n, int isign, double *tw)
{
    int nh = n / 2 > 1 ? n / 2 : 1;
    for (int k = 0; k <= nh - 1; k++) {
        double arg = 2.0 * PI * (double)k / (double)n;
        tw[2 * k] = cos(arg);
        tw[2 * k + 1] = (double)isign * sin(arg);
    }
}

/* fft3d, f90:254-304: x, then y, then z, each pencil copied to a buffer */
void ora_fft3d(double *a, int nx, int ny, int nz, int isign)
{
    if (nx > 1) {
        double *tw = malloc(sizeof(double) * 2 * (nx / 2 > 1 ? nx / 2 : 1));
        ora_twiddles(nx, isign, tw);
#pragma omp parallel
        {
            double *buf = malloc(sizeof(double) * 2 * nx);
#pragma omp for collapse(2) schedule(static)
            for (int k = 0; k < nz; k++)
                for (int j = 0; j < ny; j++) {
                    double *p = a + 2 * ((size_t)nx * (j + (size_t)ny * k));
                    memcpy(buf, p, sizeof(double) * 2 * nx);
                    ora_fft1d(buf, nx, tw);
                    memcpy(p, buf, sizeof(double) * 2 * nx);
                }
            free(buf);
        }
        free(tw);
    }
    if (ny > 1) {
        double *tw = malloc(sizeof(double) * 2 * (ny / 2 > 1 ? ny / 2 : 1));
        ora_twiddles(ny, isign, tw);
#pragma omp parallel
        {
            double *buf = malloc(sizeof(double) * 2 * ny);
#pragma omp for collapse(2) schedule(static)
            for (int k = 0; k < nz; k++)
                for (int i = 0; i < nx; i++) {
                    for (int j = 0; j < ny; j++) {
                        size_t o = 2 * (i + (size_t)nx * (j + (size_t)ny * k));
                        buf[2 * j] = a[o];
                        buf[2 * j + 1] = a[o + 1];
                    }
                    ora_fft1d(buf, ny, tw);
                    for (int j = 0; j < ny; j++) {
                        size_t o = 2 * (i + (size_t)nx * (j + (size_t)ny * k));
                        a[o] = buf[2 * j];
                        a[o + 1] = buf[2 * j + 1];
                    }
                }
            free(buf);
        }
        free(tw);
    }
    if (nz > 1) {
        double *tw = malloc(sizeof(double) * 2 * (nz / 2 > 1 ? nz / 2 : 1));
        ora_twiddles(nz, isign, tw);
#pragma omp parallel
        {
            double *buf = malloc(sizeof(double) * 2 * nz);
#pragma omp for collapse(2) schedule(static)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    for (int k = 0; k < nz; k++) {
                        size_t o = 2 * (i + (size_t)nx * (j + (size_t)ny * k));
                        buf[2 * k] = a[o];
                        buf[2 * k + 1] = a[o + 1];
                    }
                    ora_fft1d(buf, nz, tw);
                    for (int k = 0; k < nz; k++) {
                        size_t o = 2 * (i + (size_t)nx * (j + (size_t)ny * k));
                        a[o] = buf[2 * k];
                        a[o + 1] = buf[2 * k + 1];
                    }
                }
            free(buf);
        }
        free(tw);
    }
}

/* ------------------------------------------------------------------ spectrum */

/* covariance grid, forward FFT, /ntot, clip + sqrt: f90:1256-1292 */
int ora_spectrum(const ora_struct *st, int nst, double nugget, const double d[3], const int np[3],
                 double *amp, ora_spec_stats *stats)
{
    int npx = np[0], npy = np[1], npz = np[2];
    size_t ntot = (size_t)npx * npy * npz;
    double *c = malloc(sizeof(double) * 2 * ntot);
    if (!c) return 2;
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = 1; k <= npz; k++)
        for (int j = 1; j <= npy; j++)
            for (int i = 1; i <= npx; i++) {
                int kp = k - 1;
                if (kp > npz / 2) kp = kp - npz;
                int jp = j - 1;
                if (jp > npy / 2) jp = jp - npy;
                int ip = i - 1;
                if (ip > npx / 2) ip = ip - npx;
                size_t o = (size_t)(i - 1) + (size_t)npx * ((size_t)(j - 1) + (size_t)npy * (k - 1));
                c[2 * o] = ora_covariance(st, nst, nugget, (double)ip * d[0], (double)jp * d[1], (double)kp * d[2]);
                c[2 * o + 1] = 0.0;
            }
    double c0 = c[0];
    ora_fft3d(c, npx, npy, npz, -1);
    double rn = (double)ntot;
    double maximag = 0.0, maxreal = 0.0, sneg = 0.0, spos = 0.0;
    for (size_t o = 0; o < ntot; o++) {
        double re = c[2 * o] / rn;
        double im = c[2 * o + 1] / rn;
        double a = re;
        maximag = fmax(maximag, fabs(im));
        maxreal = fmax(maxreal, fabs(a));
        if (a < 0.0) {
            sneg = sneg + a;
            amp[o] = 0.0;
        } else {
            spos = spos + a;
            amp[o] = sqrt(a);
        }
    }
    free(c);
    if (stats) {
        stats->c0 = c0;
        stats->maximag = maximag;
        stats->maxreal = maxreal;
        stats->spos = spos;
        stats->sneg = sneg;
    }
    return 0;
}

/* ------------------------------------------------------------------ realizations */

/* Hermitian coefficient fill of one realization, f90:1306-1334 */
void ora_fill_coefficients(const double *amp, const int np[3], int igauss, double *c)
{
    int npx = np[0], npy = np[1], npz = np[2];
    const double s05 = sqrt(0.5);
    for (int k = 0; k <= npz - 1; k++)
        for (int j = 0; j <= npy - 1; j++)
            for (int i = 0; i <= npx - 1; i++) {
                int ip = (npx - i) % npx, jp = (npy - j) % npy, kp = (npz - k) % npz;
                long lin = i + (long)npx * (j + (long)npy * k);
                long linp = ip + (long)npx * (jp + (long)npy * kp);
                if (lin < linp) {
                    if (igauss == 1) {
                        double g1, g2;
                        ora_gauss_pair(&g1, &g2);
                        double a = amp[lin], b = amp[linp];
                        c[2 * lin] = a * g1 * s05;
                        c[2 * lin + 1] = a * g2 * s05;
                        c[2 * linp] = b * g1 * s05;
                        c[2 * linp + 1] = b * (-g2) * s05;
                    } else {
                        double phi = 2.0 * PI * ora_urand();
                        double cp = cos(phi), sp = sin(phi);
                        double a = amp[lin], b = amp[linp];
                        c[2 * lin] = a * cp;
                        c[2 * lin + 1] = a * sp;
                        c[2 * linp] = b * cp;
                        c[2 * linp + 1] = b * (-sp);
                    }
                } else if (lin == linp) {
                    if (igauss == 1) {
                        double g1, g2;
                        ora_gauss_pair(&g1, &g2);
                        c[2 * lin] = amp[lin] * g1;
                        c[2 * lin + 1] = 0.0;
                    } else if (ora_urand() < 0.5) {
                        c[2 * lin] = amp[lin];
                        c[2 * lin + 1] = 0.0;
                    } else {
                        c[2 * lin] = -amp[lin];
                        c[2 * lin + 1] = 0.0;
                    }
                }
            }
}

/* RNG states of the fill above (state after the first draw of each index) */
void ora_fill_states(const int np[3], int igauss, int64_t *first_state)
{
    int npx = np[0], npy = np[1], npz = np[2];
    for (int k = 0; k <= npz - 1; k++)
        for (int j = 0; j <= npy - 1; j++)
            for (int i = 0; i <= npx - 1; i++) {
                int ip = (npx - i) % npx, jp = (npy - j) % npy, kp = (npz - k) % npz;
                long lin = i + (long)npx * (j + (long)npy * k);
                long linp = ip + (long)npx * (jp + (long)npy * kp);
                if (lin <= linp) {
                    (void)ora_urand();
                    first_state[lin] = rng_state;
                    if (lin < linp) first_state[linp] = 0;
                    if (igauss == 1) (void)ora_urand();
                }
            }
}

/* realizations, f90:1302-1345 */
int ora_realize(const double *amp, const int np[3], const int n[3], int iseed, int nreal, int igauss,
                double *res, double *zstats)
{
    return ora_realize_range(amp, np, n, iseed, 0, nreal, igauss, res, zstats);
}

/* Realizations r_first+1 .. r_first+nreal (1-based) of the run: the stream is
 * seeded once (f90:1302-1303) and the fills of the first r_first realizations
 * are drawn and discarded (f90:1300-1334 without their transforms), so the
 * draws of every kept realization are those of the full serial run. */
int ora_realize_range(const double *amp, const int np[3], const int n[3], int iseed, int r_first, int nreal,
                      int igauss, double *res, double *zstats)
{
    int npx = np[0], npy = np[1], npz = np[2];
    int nx = n[0], ny = n[1], nz = n[2];
    size_t ntot = (size_t)npx * npy * npz;
    size_t m = (size_t)nx * ny * nz;
    double *c = malloc(sizeof(double) * 2 * ntot);
    if (!c) return 2;
    ora_rng_seed(iseed);
    for (int r = 0; r < r_first; r++) ora_fill_coefficients(amp, np, igauss, c);
    for (int r = 0; r < nreal; r++) {
        ora_fill_coefficients(amp, np, igauss, c);
        ora_fft3d(c, npx, npy, npz, +1);
        double maximag = 0.0;
        double *out = res + (size_t)r * m;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    size_t o = i + (size_t)npx * (j + (size_t)npy * k);
                    maximag = fmax(maximag, fabs(c[2 * o + 1]));
                    out[i + (size_t)nx * (j + (size_t)ny * k)] = c[2 * o];
                }
        if (zstats) {
            double s = 0.0;
            for (size_t q = 0; q < m; q++) s = s + out[q];
            double zmean = s / (double)(nx * ny * nz);
            double v = 0.0;
            for (size_t q = 0; q < m; q++) v = v + (out[q] - zmean) * (out[q] - zmean);
            zstats[3 * r] = zmean;
            zstats[3 * r + 1] = v / (double)(nx * ny * nz);
            zstats[3 * r + 2] = maximag;
        }
    }
    free(c);
    return 0;
}

/* ------------------------------------------------------------------ variogram */

/* npair_count, f90:394-402 */
int64_t ora_npair_count(int nx, int ny, int nz, int lx, int ly, int lz)
{
    if (abs(lx) >= nx || abs(ly) >= ny || abs(lz) >= nz) return 0;
    return (int64_t)(nx - abs(lx)) * (int64_t)(ny - abs(ly)) * (int64_t)(nz - abs(lz));
}

/* vario_lag, f90:405-431 (1-based loop bounds kept) */
double ora_vario_lag(const double *f, int nx, int ny, int nz, int lx, int ly, int lz)
{
    int64_t np = ora_npair_count(nx, ny, nz, lx, ly, lz);
    if (np == 0) return 0.0;
    int i0 = 1 > 1 - lx ? 1 : 1 - lx, i1 = nx < nx - lx ? nx : nx - lx;
    int j0 = 1 > 1 - ly ? 1 : 1 - ly, j1 = ny < ny - ly ? ny : ny - ly;
    int k0 = 1 > 1 - lz ? 1 : 1 - lz, k1 = nz < nz - lz ? nz : nz - lz;
    double acc = 0.0;
    for (int k = k0; k <= k1; k++)
        for (int j = j0; j <= j1; j++)
            for (int i = i0; i <= i1; i++) {
                double a = f[(i + lx - 1) + (size_t)nx * ((j + ly - 1) + (size_t)ny * (k + lz - 1))];
                double b = f[(i - 1) + (size_t)nx * ((j - 1) + (size_t)ny * (k - 1))];
                double dd = a - b;
                acc = acc + dd * dd;
            }
    return 0.5 * acc / (double)np;
}

/* task loop of vario_report, f90:462-480; gam(nlagmax, ndir, nreal) column-major */
void ora_vario_all(const double *res, const int n[3], int nreal, int ndir, const int *sx, const int *sy,
                   const int *sz, const int *nlag, double *gam)
{
    int nlagmax = 0, ntask = 0;
    for (int d = 0; d < ndir; d++) {
        if (nlag[d] > nlagmax) nlagmax = nlag[d];
        ntask += nlag[d];
    }
    int *tid = malloc(sizeof(int) * (ntask > 0 ? ntask : 1));
    int *tlag = malloc(sizeof(int) * (ntask > 0 ? ntask : 1));
    int t = 0;
    for (int d = 0; d < ndir; d++)
        for (int il = 1; il <= nlag[d]; il++) {
            tid[t] = d;
            tlag[t] = il;
            t++;
        }
    memset(gam, 0, sizeof(double) * (size_t)nlagmax * ndir * nreal);
    size_t m = (size_t)n[0] * n[1] * n[2];
    for (int r = 0; r < nreal; r++) {
#pragma omp parallel for schedule(dynamic)
        for (int q = 0; q < ntask; q++) {
            int d = tid[q], il = tlag[q];
            gam[(il - 1) + (size_t)nlagmax * (d + (size_t)ndir * r)] =
                ora_vario_lag(res + m * r, n[0], n[1], n[2], il * sx[d], il * sy[d], il * sz[d]);
        }
    }
    free(tid);
    free(tlag);
}

/* ------------------------------------------------------------------ GSLIB helpers */

static const double SQRT2 = 1.4142135623730951;   /* f90:551 */
static const double SQRT2PI = 2.5066282746310002; /* f90:552 */

/* gcum, f90:557-561 */
double ora_gcum(double x) { return 0.5 * erfc(-x / SQRT2); }

/* gauinv, f90:564-590 (Acklam rational approximation + one Halley step) */
double ora_gauinv(double p0)
{
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    double p = fmin(fmax(p0, 1.0e-15), 1.0 - 1.0e-15);
    double x, q, r;
    if (p < 0.02425) {
        q = sqrt(-2.0 * log(p));
        x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
            ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
    } else if (p <= 1.0 - 0.02425) {
        q = p - 0.5;
        r = q * q;
        x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
            (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
    } else {
        q = sqrt(-2.0 * log(1.0 - p));
        x = -((((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
              ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0));
    }
    double e = 0.5 * erfc(-x / SQRT2) - p;
    double u = e * SQRT2PI * exp(0.5 * x * x);
    x = x - u / (1.0 + 0.5 * x * u);
    return x;
}

/* heapsort_idx, f90:593-625; idx holds 1-based indices, key is 0-based storage */
static void sift(const double *key, int *idx, int root, int last)
{
    int parent = root;
    int v = idx[parent - 1];
    for (;;) {
        int child = 2 * parent;
        if (child > last) break;
        if (child < last) {
            if (key[idx[child] - 1] > key[idx[child - 1] - 1]) child = child + 1;
        }
        if (key[idx[child - 1] - 1] > key[v - 1]) {
            idx[parent - 1] = idx[child - 1];
            parent = child;
        } else {
            break;
        }
    }
    idx[parent - 1] = v;
}

void ora_heapsort_idx(const double *key, int *idx, int n)
{
    for (int i = n / 2; i >= 1; i--) sift(key, idx, i, n);
    for (int i = n; i >= 2; i--) {
        int tmp = idx[0];
        idx[0] = idx[i - 1];
        idx[i - 1] = tmp;
        sift(key, idx, 1, i - 1);
    }
}

/* powint, f90:628-636 */
static double powint(double xlow, double xhigh, double ylow, double yhigh, double xval, double pw)
{
    if (xhigh - xlow < 1.0e-20) return 0.5 * (ylow + yhigh);
    return ylow + (yhigh - ylow) * pow((xval - xlow) / (xhigh - xlow), pw);
}

/* nscore, f90:639-658 */
void ora_nscore(int nd, const double *v, const double *w, double *g, int *nt, double *vr, double *gt)
{
    int *idx = malloc(sizeof(int) * nd);
    for (int i = 0; i < nd; i++) idx[i] = i + 1;
    ora_heapsort_idx(v, idx, nd);
    double sw = 0.0;
    for (int i = 0; i < nd; i++) sw = sw + w[i];
    double cp = 0.0, oldcp = 0.0;
    for (int i = 0; i < nd; i++) {
        cp = cp + w[idx[i] - 1] / sw;
        gt[i] = ora_gauinv(0.5 * (cp + oldcp));
        vr[i] = v[idx[i] - 1];
        g[idx[i] - 1] = gt[i];
        oldcp = cp;
    }
    *nt = nd;
    free(idx);
}

/* backtr, f90:661-697 (vr, gt 0-based storage of the 1-based tables) */
double ora_backtr(double y, int nt, const double *vr, const double *gt, double zmin, double zmax,
                  int lt, double ltp, int ut, double utp)
{
    double z;
    if (y <= gt[0]) {
        double cdflo = ora_gcum(gt[0]), cdfbt = ora_gcum(y);
        if (lt == 2)
            z = powint(0.0, cdflo, zmin, vr[0], cdfbt, ltp);
        else
            z = powint(0.0, cdflo, zmin, vr[0], cdfbt, 1.0);
        if (nt == 1) z = vr[0];
    } else if (y >= gt[nt - 1]) {
        double cdfhi = ora_gcum(gt[nt - 1]), cdfbt = ora_gcum(y);
        if (ut == 2) {
            z = powint(cdfhi, 1.0, vr[nt - 1], zmax, cdfbt, utp);
        } else if (ut == 4) {
            double lam = pow(vr[nt - 1], utp) * (1.0 - cdfhi);
            z = pow(lam / fmax(1.0 - cdfbt, 1.0e-300), 1.0 / utp);
        } else {
            z = powint(cdfhi, 1.0, vr[nt - 1], zmax, cdfbt, 1.0);
        }
    } else {
        int lo = 1, hi = nt;
        while (hi - lo > 1) {
            int mid = (lo + hi) / 2;
            if (gt[mid - 1] <= y)
                lo = mid;
            else
                hi = mid;
        }
        z = powint(gt[lo - 1], gt[hi - 1], vr[lo - 1], vr[hi - 1], y, 1.0);
    }
    return z;
}

/* ------------------------------------------------------------------ conditioning */

static int fnint(double x) { return (int)lround(x); } /* Fortran nint: half away from zero */

typedef struct {
    const ora_struct *st;
    int nst;
    double nugget;
    ora_struct srch;
    double rmax;
    int nx, ny, nz, nreal, ndmax;
    double xmin, ymin, zmin, dx, dy, dz;
    int nsbx, nsby, nsbz, mbx, mby, mbz;
    double bsx, bsy, bsz, c0;
    const int *sbstart, *sbidx;
    const int *ix, *iy, *iz;
    const double *dxs, *dys, *dzs, *dg, *simd;
    int nd;
    double *res;
} cond_ctx;

/* chol_solve, f90:1040-1079; a, lmat are ndmax x ndmax column-major */
static void chol_solve(const double *a, const double *bvec, double *wgt, int n, int ld, double ridge, int *ok,
                       double *lmat)
{
#define A(p, q) a[((p)-1) + (size_t)ld * ((q)-1)]
#define L(p, q) lmat[((p)-1) + (size_t)ld * ((q)-1)]
    *ok = 1;
    for (int p = 1; p <= n; p++) {
        for (int q = 1; q <= p; q++) {
            double s = A(p, q);
            if (p == q) s = s + ridge;
            for (int m = 1; m <= q - 1; m++) s = s - L(p, m) * L(q, m);
            if (p == q) {
                if (s <= 0.0) {
                    *ok = 0;
                    return;
                }
                L(p, p) = sqrt(s);
            } else {
                L(p, q) = s / L(q, q);
            }
        }
    }
    for (int p = 1; p <= n; p++) {
        double s = bvec[p - 1];
        for (int m = 1; m <= p - 1; m++) s = s - L(p, m) * wgt[m - 1];
        wgt[p - 1] = s / L(p, p);
    }
    for (int p = n; p >= 1; p--) {
        double s = wgt[p - 1];
        for (int m = p + 1; m <= n; m++) s = s - L(m, p) * wgt[m - 1];
        wgt[p - 1] = s / L(p, p);
    }
#undef A
#undef L
}

/* krige_node, f90:949-1038 */
static void krige_node(const cond_ctx *cx, int i, int j, int k, int64_t *nsum, int *nfail, int *nnone, int *nexact,
                       double *cd, int *cid, double *a, double *bvec, double *wgt, double *lmat)
{
    int ndmax = cx->ndmax;
    double x = cx->xmin + (double)(i - 1) * cx->dx;
    double y = cx->ymin + (double)(j - 1) * cx->dy;
    double z = cx->zmin + (double)(k - 1) * cx->dz;
    int bx = (int)((x - cx->xmin + 0.5 * cx->dx) / cx->bsx) + 1;
    bx = bx < 1 ? 1 : bx;
    bx = bx > cx->nsbx ? cx->nsbx : bx;
    int by = (int)((y - cx->ymin + 0.5 * cx->dy) / cx->bsy) + 1;
    by = by < 1 ? 1 : by;
    by = by > cx->nsby ? cx->nsby : by;
    int bz = (int)((z - cx->zmin + 0.5 * cx->dz) / cx->bsz) + 1;
    bz = bz < 1 ? 1 : bz;
    bz = bz > cx->nsbz ? cx->nsbz : bz;
    const double (*R)[3] = cx->srch.rot;
    double rm2 = cx->rmax * cx->rmax;
    int nn = 0;
    int kb0 = bz - cx->mbz > 1 ? bz - cx->mbz : 1, kb1 = bz + cx->mbz < cx->nsbz ? bz + cx->mbz : cx->nsbz;
    int jb0 = by - cx->mby > 1 ? by - cx->mby : 1, jb1 = by + cx->mby < cx->nsby ? by + cx->mby : cx->nsby;
    int ib0 = bx - cx->mbx > 1 ? bx - cx->mbx : 1, ib1 = bx + cx->mbx < cx->nsbx ? bx + cx->mbx : cx->nsbx;
    for (int kb = kb0; kb <= kb1; kb++)
        for (int jb = jb0; jb <= jb1; jb++)
            for (int ib = ib0; ib <= ib1; ib++) {
                int blk = ib + cx->nsbx * (jb - 1 + cx->nsby * (kb - 1));
                for (int p = cx->sbstart[blk - 1]; p <= cx->sbstart[blk] - 1; p++) {
                    int q = cx->sbidx[p - 1];
                    double hx = cx->dxs[q - 1] - x, hy = cx->dys[q - 1] - y, hz = cx->dzs[q - 1] - z;
                    double rx = R[0][0] * hx + R[0][1] * hy + R[0][2] * hz;
                    double ry = R[1][0] * hx + R[1][1] * hy + R[1][2] * hz;
                    double rz = R[2][0] * hx + R[2][1] * hy + R[2][2] * hz;
                    double d2 = (rx * rx + ry * ry + rz * rz) / rm2;
                    if (d2 > 1.0) continue;
                    int m;
                    if (nn < ndmax) {
                        nn = nn + 1;
                        m = nn;
                    } else if (d2 < cd[nn - 1]) {
                        m = nn;
                    } else {
                        continue;
                    }
                    while (m > 1) {
                        if (cd[m - 2] <= d2) break;
                        cd[m - 1] = cd[m - 2];
                        cid[m - 1] = cid[m - 2];
                        m = m - 1;
                    }
                    cd[m - 1] = d2;
                    cid[m - 1] = q;
                }
            }
    *nsum += nn;
    size_t m3 = (size_t)cx->nx * cx->ny * cx->nz;
    size_t node = (size_t)(i - 1) + (size_t)cx->nx * ((size_t)(j - 1) + (size_t)cx->ny * (k - 1));
    if (nn == 0) {
        *nnone += 1;
        return;
    }
    if (cd[0] == 0.0) {
        int q = cid[0];
        if (cx->ix[q - 1] == i && cx->iy[q - 1] == j && cx->iz[q - 1] == k) {
            for (int l = 0; l < cx->nreal; l++) cx->res[node + m3 * l] = cx->dg[q - 1];
            *nexact += 1;
            return;
        }
    }
    for (int p = 1; p <= nn; p++) {
        int cp = cid[p - 1];
        for (int q = 1; q <= p; q++) {
            int cq = cid[q - 1];
            double v = ora_covariance(cx->st, cx->nst, cx->nugget, cx->dxs[cp - 1] - cx->dxs[cq - 1],
                                      cx->dys[cp - 1] - cx->dys[cq - 1], cx->dzs[cp - 1] - cx->dzs[cq - 1]);
            a[(p - 1) + (size_t)ndmax * (q - 1)] = v;
            a[(q - 1) + (size_t)ndmax * (p - 1)] = v;
        }
        bvec[p - 1] = ora_covariance(cx->st, cx->nst, cx->nugget, cx->dxs[cp - 1] - x, cx->dys[cp - 1] - y,
                                     cx->dzs[cp - 1] - z);
    }
    double ridge = 1.0e-10 * cx->c0;
    int ok = 0, jj;
    for (jj = 1; jj <= 3; jj++) {
        chol_solve(a, bvec, wgt, nn, ndmax, ridge, &ok, lmat);
        if (ok) break;
        ridge = ridge * 1.0e3;
    }
    if (!ok) {
        *nfail += 1;
        return;
    }
    if (jj > 1) *nfail += 1;
    double zk = 0.0;
    for (int p = 1; p <= nn; p++) zk = zk + wgt[p - 1] * cx->dg[cid[p - 1] - 1];
    for (int l = 0; l < cx->nreal; l++) {
        double sks = 0.0;
        for (int p = 1; p <= nn; p++) sks = sks + wgt[p - 1] * cx->simd[(cid[p - 1] - 1) + (size_t)cx->nd * l];
        cx->res[node + m3 * l] = zk + cx->res[node + m3 * l] - sks;
    }
}

/* condition_field after the parameter/data reading, f90:782-924 */
int ora_condition(double *res, const int n[3], int nreal, const double xmin3[3], const double d[3],
                  const ora_struct *st, int nst, double nugget, const ora_cond_params *cp,
                  const double *raw_rows, int nrows, int nvar, ora_cond_stats *cs,
                  double *vrt_out, double *gtt_out, double *dxs_out, double *dys_out, double *dzs_out,
                  double *dval_out, double *dg_out)
{
    int nx = n[0], ny = n[1], nz = n[2];
    double xmin = xmin3[0], ymin = xmin3[1], zmin = xmin3[2];
    double dx = d[0], dy = d[1], dz = d[2];
    ora_struct srch;
    memset(&srch, 0, sizeof srch);
    srch.itype = 1;
    srch.sill = 1.0;
    srch.ahmax = cp->rmax;
    srch.ahmin = cp->rmed;
    srch.avert = cp->rvert;
    srch.az = cp->sa1;
    srch.dip = cp->sa2;
    srch.plg = cp->sa3;
    ora_setrot(&srch);
    double ex = sqrt(srch.axes[0][0] * srch.axes[0][0] + srch.axes[1][0] * srch.axes[1][0] +
                     srch.axes[2][0] * srch.axes[2][0]);
    double ey = sqrt(srch.axes[0][1] * srch.axes[0][1] + srch.axes[1][1] * srch.axes[1][1] +
                     srch.axes[2][1] * srch.axes[2][1]);
    double ez = sqrt(srch.axes[0][2] * srch.axes[0][2] + srch.axes[1][2] * srch.axes[1][2] +
                     srch.axes[2][2] * srch.axes[2][2]);

    /* data snapping, f90:782-802 */
    double *raw = malloc(sizeof(double) * 5 * (nrows > 0 ? nrows : 1));
    double *key = malloc(sizeof(double) * (nrows > 0 ? nrows : 1));
    int nn = 0, nout = 0;
    for (int q = 0; q < nrows; q++) {
        const double *row = raw_rows + (size_t)q * nvar;
        double v = row[cp->ivc - 1];
        if (v < cp->tmin || v >= cp->tmax) continue;
        int j = fnint((row[cp->ixc - 1] - xmin) / dx) + 1;
        int k = fnint((row[cp->iyc - 1] - ymin) / dy) + 1;
        int r = 1;
        if (cp->izc > 0 && nz > 1) r = fnint((row[cp->izc - 1] - zmin) / dz) + 1;
        if (j < 1 || j > nx || k < 1 || k > ny || r < 1 || r > nz) {
            nout++;
            continue;
        }
        double *o = raw + 5 * (size_t)nn;
        o[0] = (double)j;
        o[1] = (double)k;
        o[2] = (double)r;
        o[3] = v;
        o[4] = 1.0;
        if (cp->iwc > 0) o[4] = row[cp->iwc - 1];
        key[nn] = (double)j + (double)nx * ((double)(k - 1) + (double)ny * (double)(r - 1));
        nn++;
    }
    if (nn == 0) {
        free(raw);
        free(key);
        return 3;
    }
    /* merge data of the same node, f90:805-828 */
    int *ord = malloc(sizeof(int) * nn);
    for (int q = 0; q < nn; q++) ord[q] = q + 1;
    ora_heapsort_idx(key, ord, nn);
    int *ix = malloc(sizeof(int) * nn), *iy = malloc(sizeof(int) * nn), *iz = malloc(sizeof(int) * nn);
    double *dval = malloc(sizeof(double) * nn), *dwt = malloc(sizeof(double) * nn);
    int nd = 0;
    int i = 1;
    while (i <= nn) {
        int j = i;
        while (j < nn) {
            if (key[ord[j] - 1] != key[ord[i - 1] - 1]) break;
            j = j + 1;
        }
        ix[nd] = fnint(raw[5 * (ord[i - 1] - 1) + 0]);
        iy[nd] = fnint(raw[5 * (ord[i - 1] - 1) + 1]);
        iz[nd] = fnint(raw[5 * (ord[i - 1] - 1) + 2]);
        double sw = 0.0, svw = 0.0;
        for (int q = i; q <= j; q++) sw = sw + raw[5 * (ord[q - 1] - 1) + 4];
        for (int q = i; q <= j; q++) svw = svw + raw[5 * (ord[q - 1] - 1) + 3] * raw[5 * (ord[q - 1] - 1) + 4];
        dwt[nd] = sw;
        dval[nd] = svw / dwt[nd];
        nd++;
        i = j + 1;
    }
    int nmerged = nn - nd;
    double *dxs = malloc(sizeof(double) * nd), *dys = malloc(sizeof(double) * nd), *dzs = malloc(sizeof(double) * nd);
    double *dg = malloc(sizeof(double) * nd);
    for (int q = 0; q < nd; q++) {
        dxs[q] = xmin + (double)(ix[q] - 1) * dx;
        dys[q] = ymin + (double)(iy[q] - 1) * dy;
        dzs[q] = zmin + (double)(iz[q] - 1) * dz;
    }
    /* normal scores, f90:830-847 */
    double *vrt = malloc(sizeof(double) * nd), *gtt = malloc(sizeof(double) * nd);
    int nt = nd;
    if (cp->itrans == 1) {
        ora_nscore(nd, dval, dwt, dg, &nt, vrt, gtt);
    } else {
        for (int q = 0; q < nd; q++) dg[q] = dval[q] - cp->skmean;
    }
    /* simulated values at the data nodes, f90:858-863 */
    size_t m3 = (size_t)nx * ny * nz;
    double *simd = malloc(sizeof(double) * (size_t)nd * nreal);
    for (int r = 0; r < nreal; r++)
        for (int q = 0; q < nd; q++)
            simd[q + (size_t)nd * r] =
                res[(size_t)(ix[q] - 1) + (size_t)nx * ((size_t)(iy[q] - 1) + (size_t)ny * (iz[q] - 1)) + m3 * r];
    /* super blocks, f90:866-892 */
    int nsbx = (int)ceil((double)nx * dx / (0.5 * ex));
    nsbx = nsbx > 100 ? 100 : nsbx;
    nsbx = nsbx < 1 ? 1 : nsbx;
    int nsby = (int)ceil((double)ny * dy / (0.5 * ey));
    nsby = nsby > 100 ? 100 : nsby;
    nsby = nsby < 1 ? 1 : nsby;
    int nsbz = (int)ceil((double)nz * dz / (0.5 * ez));
    nsbz = nsbz > 100 ? 100 : nsbz;
    nsbz = nsbz < 1 ? 1 : nsbz;
    if (nz == 1) nsbz = 1;
    while ((double)nsbx * nsby * nsbz > 2.0e6) {
        nsbx = nsbx * 3 / 4 > 1 ? nsbx * 3 / 4 : 1;
        nsby = nsby * 3 / 4 > 1 ? nsby * 3 / 4 : 1;
        nsbz = nsbz * 3 / 4 > 1 ? nsbz * 3 / 4 : 1;
    }
    int nsb = nsbx * nsby * nsbz;
    double bsx = (double)nx * dx / (double)nsbx, bsy = (double)ny * dy / (double)nsby,
           bsz = (double)nz * dz / (double)nsbz;
    int mbx = (int)ceil(ex / bsx), mby = (int)ceil(ey / bsy), mbz = (int)ceil(ez / bsz);
    int *sbstart = malloc(sizeof(int) * (nsb + 1)), *sbcount = calloc(nsb, sizeof(int));
    int *sbidx = malloc(sizeof(int) * nd), *sbof = malloc(sizeof(int) * nd);
    for (int q = 0; q < nd; q++) {
        int b1 = (int)((dxs[q] - xmin + 0.5 * dx) / bsx) + 1;
        b1 = b1 < 1 ? 1 : b1;
        b1 = b1 > nsbx ? nsbx : b1;
        int b2 = (int)((dys[q] - ymin + 0.5 * dy) / bsy) + 1;
        b2 = b2 < 1 ? 1 : b2;
        b2 = b2 > nsby ? nsby : b2;
        int b3 = (int)((dzs[q] - zmin + 0.5 * dz) / bsz) + 1;
        b3 = b3 < 1 ? 1 : b3;
        b3 = b3 > nsbz ? nsbz : b3;
        sbof[q] = b1 + nsbx * (b2 - 1 + nsby * (b3 - 1));
        sbcount[sbof[q] - 1]++;
    }
    sbstart[0] = 1;
    for (int q = 1; q <= nsb; q++) sbstart[q] = sbstart[q - 1] + sbcount[q - 1];
    memset(sbcount, 0, sizeof(int) * nsb);
    for (int q = 0; q < nd; q++) {
        int b = sbof[q];
        sbidx[sbstart[b - 1] + sbcount[b - 1] - 1] = q + 1;
        sbcount[b - 1]++;
    }
    cond_ctx cx;
    cx.st = st;
    cx.nst = nst;
    cx.nugget = nugget;
    cx.srch = srch;
    cx.rmax = cp->rmax;
    cx.nx = nx;
    cx.ny = ny;
    cx.nz = nz;
    cx.nreal = nreal;
    cx.ndmax = cp->ndmax;
    cx.xmin = xmin;
    cx.ymin = ymin;
    cx.zmin = zmin;
    cx.dx = dx;
    cx.dy = dy;
    cx.dz = dz;
    cx.nsbx = nsbx;
    cx.nsby = nsby;
    cx.nsbz = nsbz;
    cx.mbx = mbx;
    cx.mby = mby;
    cx.mbz = mbz;
    cx.bsx = bsx;
    cx.bsy = bsy;
    cx.bsz = bsz;
    cx.c0 = ora_covariance(st, nst, nugget, 0.0, 0.0, 0.0);
    cx.sbstart = sbstart;
    cx.sbidx = sbidx;
    cx.ix = ix;
    cx.iy = iy;
    cx.iz = iz;
    cx.dxs = dxs;
    cx.dys = dys;
    cx.dzs = dzs;
    cx.dg = dg;
    cx.simd = simd;
    cx.nd = nd;
    cx.res = res;
    /* kriging of the residual at every node, f90:895-906 */
    int64_t nsum = 0;
    int nfail = 0, nnone = 0, nexact = 0;
    int ndmax = cp->ndmax;
#pragma omp parallel reduction(+ : nsum, nfail, nnone, nexact)
    {
        double *cd = malloc(sizeof(double) * ndmax);
        int *cid = malloc(sizeof(int) * ndmax);
        double *a = malloc(sizeof(double) * ndmax * ndmax);
        double *lmat = malloc(sizeof(double) * ndmax * ndmax);
        double *bvec = malloc(sizeof(double) * ndmax), *wgt = malloc(sizeof(double) * ndmax);
#pragma omp for collapse(2) schedule(dynamic, 2)
        for (int k = 1; k <= nz; k++)
            for (int j = 1; j <= ny; j++)
                for (int ii = 1; ii <= nx; ii++)
                    krige_node(&cx, ii, j, k, &nsum, &nfail, &nnone, &nexact, cd, cid, a, bvec, wgt, lmat);
        free(cd);
        free(cid);
        free(a);
        free(lmat);
        free(bvec);
        free(wgt);
    }
    /* back transform or mean restore, f90:909-924 */
    if (cp->itrans == 1) {
#pragma omp parallel for schedule(static)
        for (long q = 0; q < (long)(m3 * nreal); q++)
            res[q] = ora_backtr(res[q], nt, vrt, gtt, cp->zlo, cp->zhi, cp->ltail, cp->ltpar, cp->utail, cp->utpar);
    } else if (cp->skmean != 0.0) {
        for (size_t q = 0; q < m3 * nreal; q++) res[q] = res[q] + cp->skmean;
    }
    if (cs) {
        cs->nd = nd;
        cs->nmerged = nmerged;
        cs->nout = nout;
        cs->nsb[0] = nsbx;
        cs->nsb[1] = nsby;
        cs->nsb[2] = nsbz;
        cs->nsum = nsum;
        cs->nfail = nfail;
        cs->nnone = nnone;
        cs->nexact = nexact;
    }
    for (int q = 0; q < nd; q++) {
        if (vrt_out) vrt_out[q] = vrt[q];
        if (gtt_out) gtt_out[q] = gtt[q];
        if (dxs_out) dxs_out[q] = dxs[q];
        if (dys_out) dys_out[q] = dys[q];
        if (dzs_out) dzs_out[q] = dzs[q];
        if (dval_out) dval_out[q] = dval[q];
        if (dg_out) dg_out[q] = dg[q];
    }
    free(raw);
    free(key);
    free(ord);
    free(ix);
    free(iy);
    free(iz);
    free(dval);
    free(dwt);
    free(dxs);
    free(dys);
    free(dzs);
    free(dg);
    free(vrt);
    free(gtt);
    free(simd);
    free(sbstart);
    free(sbcount);
    free(sbidx);
    free(sbof);
    return 0;
}
