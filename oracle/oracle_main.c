/*
 * oracle_main.c -- command-line driver of the CPU oracle: a restatement of the
 * main program of src/specsim3d.f90 (f90:1085-1418), the variogram report
 * (f90:434-529), the conditioning reader (f90:729-855) and the writers
 * (f90:307-391, f90:1357-1414).
 *
 * TEST INFRASTRUCTURE ONLY: built as oracle/_build/specsim3d_oracle and used
 * by the tests as an independent black-box implementation of the reference
 * program (same parameter files in, same files and stdout lines out).
 */
#include "ss3d_oracle.h"

#include <ctype.h>
#include <errno.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------ Fortran edit descriptors */

static void pad_to(char *out, const char *s, int w)
{
    int n = (int)strlen(s);
    if (w <= 0) {
        strcpy(out, s);
        return;
    }
    if (n > w) {
        for (int i = 0; i < w; i++) out[i] = '*';
        out[w] = 0;
        return;
    }
    int p = w - n;
    memset(out, ' ', p);
    strcpy(out + p, s);
}

static int nonfinite(char *out, double x, int w)
{
    if (isnan(x)) {
        pad_to(out, "NaN", w);
        return 1;
    }
    if (isinf(x)) {
        const char *s = x < 0 ? (w >= 9 ? "-Infinity" : "-Inf") : (w >= 8 ? "Infinity" : "Inf");
        pad_to(out, s, w);
        return 1;
    }
    return 0;
}

/* ESw.d */
static void f_es(char *out, double x, int w, int d)
{
    if (nonfinite(out, x, w)) return;
    char buf[64], res[80];
    snprintf(buf, sizeof buf, "%.*E", d, x);
    char *e = strchr(buf, 'E');
    int ex = atoi(e + 1);
    *e = 0;
    if (x == 0.0) ex = 0;
    if (abs(ex) <= 99)
        snprintf(res, sizeof res, "%sE%c%02d", buf, ex < 0 ? '-' : '+', abs(ex));
    else
        snprintf(res, sizeof res, "%s%c%03d", buf, ex < 0 ? '-' : '+', abs(ex));
    pad_to(out, res, w);
}

/* Fw.d */
static void f_f(char *out, double x, int w, int d)
{
    if (nonfinite(out, x, w)) return;
    char buf[400];
    snprintf(buf, sizeof buf, "%.*f", d, x);
    if ((int)strlen(buf) > w) {
        if (buf[0] == '0' && buf[1] == '.')
            memmove(buf, buf + 1, strlen(buf));
        else if (buf[0] == '-' && buf[1] == '0' && buf[2] == '.')
            memmove(buf + 1, buf + 2, strlen(buf + 1));
    }
    pad_to(out, buf, w);
}

/* Iw (w = 0 gives I0) */
static void f_i(char *out, long long v, int w)
{
    char buf[32];
    snprintf(buf, sizeof buf, "%lld", v);
    pad_to(out, buf, w);
}

static const char *ES(double x, int w, int d)
{
    static char ring[16][96];
    static int slot = 0;
    char *o = ring[slot++ & 15];
    f_es(o, x, w, d);
    return o;
}
static const char *FF(double x, int w, int d)
{
    static char ring[16][420];
    static int slot = 0;
    char *o = ring[slot++ & 15];
    f_f(o, x, w, d);
    return o;
}
static const char *II(long long v, int w)
{
    static char ring[16][40];
    static int slot = 0;
    char *o = ring[slot++ & 15];
    f_i(o, v, w);
    return o;
}

static void fstop_code(int code)
{
    fflush(stdout);
    fprintf(stderr, "STOP %d\n", code);
    exit(code);
}
static void fstop_msg(const char *msg)
{
    fflush(stdout);
    fprintf(stderr, "STOP %s\n", msg);
    exit(0);
}

/* ------------------------------------------------------------------ records and list-directed input */

typedef struct {
    char **lines;
    int n, pos;
} recfile;

static int rec_open(recfile *f, const char *path, int maxlen)
{
    FILE *fp = fopen(path, "r");
    if (!fp) return 1;
    f->lines = NULL;
    f->n = 0;
    f->pos = 0;
    int cap = 0;
    char *line = NULL;
    size_t lcap = 0;
    ssize_t got;
    while ((got = getline(&line, &lcap, fp)) >= 0) {
        while (got > 0 && (line[got - 1] == '\n' || line[got - 1] == '\r')) line[--got] = 0;
        if (maxlen > 0 && got > maxlen) line[maxlen] = 0;
        if (f->n == cap) {
            cap = cap ? 2 * cap : 64;
            f->lines = realloc(f->lines, sizeof(char *) * cap);
        }
        f->lines[f->n++] = strdup(line);
    }
    free(line);
    fclose(fp);
    return 0;
}

static void rec_close(recfile *f)
{
    for (int i = 0; i < f->n; i++) free(f->lines[i]);
    free(f->lines);
    f->lines = NULL;
    f->n = 0;
}

/* formatted '(a)' read of one record: NULL at end of file */
static const char *rec_read_a(recfile *f)
{
    if (f->pos >= f->n) return NULL;
    return f->lines[f->pos++];
}

static int parse_int_tok(const char *t, long long *v)
{
    const char *p = t;
    if (*p == '+' || *p == '-') p++;
    if (!isdigit((unsigned char)*p)) return 1;
    while (isdigit((unsigned char)*p)) p++;
    if (*p) return 1;
    *v = strtoll(t, NULL, 10);
    return 0;
}

static int parse_real_tok(const char *t, double *v)
{
    char buf[128];
    size_t n = strlen(t);
    if (n >= sizeof buf) return 1;
    for (size_t i = 0; i <= n; i++) {
        char c = t[i];
        buf[i] = (c == 'd' || c == 'D' || c == 'q' || c == 'Q') ? 'e' : c;
    }
    const char *p = buf;
    if (*p == '+' || *p == '-') p++;
    int digits = 0;
    while (isdigit((unsigned char)*p)) {
        p++;
        digits++;
    }
    if (*p == '.') {
        p++;
        while (isdigit((unsigned char)*p)) {
            p++;
            digits++;
        }
    }
    if (!digits) {
        /* Infinity / NaN spellings */
        char *end;
        errno = 0;
        double x = strtod(buf, &end);
        if (end != buf && *end == 0 && (isinf(x) || isnan(x))) {
            *v = x;
            return 0;
        }
        return 1;
    }
    if (*p == 'e' || *p == 'E') {
        p++;
        if (*p == '+' || *p == '-') p++;
        if (!isdigit((unsigned char)*p)) return 1;
        while (isdigit((unsigned char)*p)) p++;
    }
    if (*p) return 1;
    *v = strtod(buf, NULL);
    return 0;
}

/* List-directed read of len(kinds) items ('i' int, 'd' double) from records,
 * continuing over records as Fortran does.  Returns 0, -1 at end of file before
 * all items were read, or 1 on a conversion error.  A '/' ends the read. */
static int ld_read(recfile *f, const char *kinds, void **out)
{
    int nitems = (int)strlen(kinds), item = 0;
    int rec = f->pos;
    while (item < nitems) {
        if (rec >= f->n) return -1;
        const char *s = f->lines[rec];
        const char *p = s;
        int prev_comma = 0;
        while (item < nitems) {
            while (*p == ' ' || *p == '\t') p++;
            if (!*p) break;
            if (*p == '/') {
                f->pos = rec + 1;
                return 0;
            }
            if (*p == ',') {
                if (prev_comma) item++; /* null value */
                prev_comma = 1;
                p++;
                continue;
            }
            const char *q = p;
            while (*q && *q != ' ' && *q != '\t' && *q != ',' && *q != '/') q++;
            char tok[128];
            size_t tl = (size_t)(q - p);
            if (tl >= sizeof tok) return 1;
            memcpy(tok, p, tl);
            tok[tl] = 0;
            p = q;
            prev_comma = 0;
            int rep = 1;
            char *star = strchr(tok, '*');
            char *val = tok;
            if (star) {
                *star = 0;
                long long r;
                if (parse_int_tok(tok, &r) || r < 1) return 1;
                rep = (int)r;
                val = star + 1;
            }
            for (int k = 0; k < rep && item < nitems; k++, item++) {
                if (!*val) continue; /* r* : null values */
                if (kinds[item] == 'i') {
                    long long v;
                    if (parse_int_tok(val, &v)) return 1;
                    *(int *)out[item] = (int)v;
                } else {
                    double v;
                    if (parse_real_tok(val, &v)) return 1;
                    *(double *)out[item] = v;
                }
            }
            while (*p == ' ' || *p == '\t') p++;
            if (*p == ',') {
                p++;
                prev_comma = 1;
            }
        }
        rec++;
    }
    f->pos = rec;
    return 0;
}

static void ld_or_die(recfile *f, const char *kinds, void **out, const char *what)
{
    int rc = ld_read(f, kinds, out);
    if (rc != 0) {
        fflush(stdout);
        fprintf(stderr, "Fortran runtime error: %s while reading %s\n", rc < 0 ? "End of file" : "Bad value", what);
        exit(2);
    }
}

static void trim_copy(char *dst, const char *src, size_t cap)
{
    while (*src == ' ' || *src == '\t') src++;
    size_t n = strlen(src);
    while (n > 0 && (src[n - 1] == ' ' || src[n - 1] == '\t')) n--;
    if (n >= cap) n = cap - 1;
    memcpy(dst, src, n);
    dst[n] = 0;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* ------------------------------------------------------------------ writers */

static void put_be32(FILE *fp, float v)
{
    unsigned char b[4], o[4];
    memcpy(b, &v, 4);
    o[0] = b[3];
    o[1] = b[2];
    o[2] = b[1];
    o[3] = b[0];
    fwrite(o, 1, 4, fp);
}

/* write_vtk_bin, f90:362-391 */
static void write_vtk_bin(const char *fname, const float *a, int nx, int ny, int nz, double x0, double y0, double z0,
                          double dx, double dy, double dz, const char *title)
{
    FILE *fp = fopen(fname, "wb");
    if (!fp) return;
    fprintf(fp, "# vtk DataFile Version 3.0\n%s\nBINARY\nDATASET STRUCTURED_POINTS\n", title);
    fprintf(fp, "DIMENSIONS %d %d %d\n", nx, ny, nz);
    fprintf(fp, "ORIGIN %s %s %s\n", ES(x0, 16, 8), ES(y0, 16, 8), ES(z0, 16, 8));
    fprintf(fp, "SPACING %s %s %s\n", ES(dx, 16, 8), ES(dy, 16, 8), ES(dz, 16, 8));
    fprintf(fp, "POINT_DATA %lld\n", (long long)nx * ny * nz);
    fprintf(fp, "SCALARS sim float 1\nLOOKUP_TABLE default\n");
    size_t m = (size_t)nx * ny * nz;
    for (size_t i = 0; i < m; i++) put_be32(fp, a[i]);
    fputc('\n', fp);
    fclose(fp);
}

/* write_vti, f90:307-359 */
static void write_vti(const char *fname, const double *res, int nx, int ny, int nz, int nreal, double x0, double y0,
                      double z0, double dx, double dy, double dz)
{
    FILE *fp = fopen(fname, "wb");
    if (!fp) return;
    long long nbytes = 4LL * nx * ny * nz;
    char ext[128];
    snprintf(ext, sizeof ext, "0 %d 0 %d 0 %d", nx - 1, ny - 1, nz - 1);
    fprintf(fp, "<?xml version=\"1.0\"?>\n");
    fprintf(fp, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
    fprintf(fp, "  <ImageData WholeExtent=\"%s\" Origin=\" %s %s %s\" Spacing=\" %s %s %s\">\n", ext, ES(x0, 16, 8),
            ES(y0, 16, 8), ES(z0, 16, 8), ES(dx, 16, 8), ES(dy, 16, 8), ES(dz, 16, 8));
    fprintf(fp, "    <Piece Extent=\"%s\">\n", ext);
    fprintf(fp, "      <PointData Scalars=\"sim_1\">\n");
    for (int r = 1; r <= nreal; r++)
        fprintf(fp, "        <DataArray type=\"Float32\" Name=\"sim_%d\" format=\"appended\" offset=\"%lld\"/>\n", r,
                (nbytes + 8) * (long long)(r - 1));
    fprintf(fp, "      </PointData>\n      <CellData/>\n    </Piece>\n  </ImageData>\n");
    fprintf(fp, "  <AppendedData encoding=\"raw\">\n   _");
    size_t m = (size_t)nx * ny * nz;
    float *sp = malloc(sizeof(float) * m);
    for (int r = 0; r < nreal; r++) {
        for (size_t i = 0; i < m; i++) sp[i] = (float)res[i + m * r];
        unsigned long long nb = (unsigned long long)nbytes;
        fwrite(&nb, 8, 1, fp);
        fwrite(sp, sizeof(float), m, fp);
    }
    free(sp);
    fprintf(fp, "\n  </AppendedData>\n</VTKFile>\n");
    fclose(fp);
}

/* ------------------------------------------------------------------ variogram report, f90:434-529 */

static void vario_report(const char *varfile, const char *outbase, const double *res, const int n[3], int nreal,
                         const double d[3], const ora_struct *st, int nst, double nugget)
{
    recfile vf;
    if (rec_open(&vf, varfile, 0)) {
        printf(" cannot open variogram file: %s\n", varfile);
        return;
    }
    int ndir = 0, iper = 0;
    void *o2[2] = {&ndir, &iper};
    ld_or_die(&vf, "ii", o2, "variogram file");
    int *sx = calloc(ndir, sizeof(int)), *sy = calloc(ndir, sizeof(int)), *sz = calloc(ndir, sizeof(int)),
        *nlag = calloc(ndir, sizeof(int));
    for (int id = 0; id < ndir; id++) {
        void *o4[4] = {&sx[id], &sy[id], &sz[id], &nlag[id]};
        ld_or_die(&vf, "iiii", o4, "variogram file");
    }
    rec_close(&vf);
    int nlagmax = 0;
    for (int id = 0; id < ndir; id++)
        if (nlag[id] > nlagmax) nlagmax = nlag[id];
    double *gam = calloc((size_t)(nlagmax > 0 ? nlagmax : 1) * ndir * nreal, sizeof(double));
    ora_vario_all(res, n, nreal, ndir, sx, sy, sz, nlag, gam);
    double c0 = nugget;
    for (int i = 0; i < nst; i++) c0 = c0 + st[i].sill;
    char fname[1100];
    snprintf(fname, sizeof fname, "%s_vario.csv", outbase);
    FILE *fp = fopen(fname, "w");
    fprintf(fp, "dir,sx,sy,sz,lag,h,npairs,gamma_model,gamma_mean,gamma_sd");
    if (iper == 1)
        for (int r = 1; r <= nreal; r++) fprintf(fp, ",gamma_r%d", r);
    fprintf(fp, "\n");
    printf(" variograms (Fortran): direction  lags  RMS(mean-model)  max|err|   [rising part, gamma_model < 0.95 sill]\n");
    for (int id = 0; id < ndir; id++) {
        double rms = 0.0, mx = 0.0;
        int nfit = 0;
        for (int il = 1; il <= nlag[id]; il++) {
            int64_t np = ora_npair_count(n[0], n[1], n[2], il * sx[id], il * sy[id], il * sz[id]);
            if (np == 0) continue;
            double hx = (double)(il * sx[id]) * d[0], hy = (double)(il * sy[id]) * d[1],
                   hz = (double)(il * sz[id]) * d[2];
            double h = sqrt(hx * hx + hy * hy + hz * hz);
            double gth = c0 - ora_covariance(st, nst, nugget, hx, hy, hz);
            const double *g = gam + (il - 1) + (size_t)nlagmax * id;
            size_t gs = (size_t)nlagmax * ndir;
            double s = 0.0;
            for (int r = 0; r < nreal; r++) s = s + g[gs * r];
            double gm = s / (double)nreal;
            double gsd = 0.0;
            if (nreal > 1) {
                double v = 0.0;
                for (int r = 0; r < nreal; r++) v = v + (g[gs * r] - gm) * (g[gs * r] - gm);
                gsd = sqrt(v / (double)(nreal - 1));
            }
            fprintf(fp, "%d,%d,%d,%d,%d,%s,%lld,%s,%s,%s", id + 1, sx[id], sy[id], sz[id], il, ES(h, 14, 6),
                    (long long)np, ES(gth, 14, 6), ES(gm, 14, 6), ES(gsd, 14, 6));
            if (iper == 1)
                for (int r = 0; r < nreal; r++) fprintf(fp, ",%s", ES(g[gs * r], 14, 6));
            fprintf(fp, "\n");
            if (gth < 0.95 * c0) {
                double e = gm - gth;
                rms = rms + e * e;
                mx = fmax(mx, fabs(e));
                nfit++;
            }
        }
        if (nfit > 0) rms = sqrt(rms / (double)nfit);
        printf("   dir%s%s%s%s%s%s%s\n", II(id + 1, 3), II(sx[id], 4), II(sy[id], 4), II(sz[id], 4), II(nlag[id], 6),
               FF(rms, 12, 5), FF(mx, 12, 5));
    }
    fclose(fp);
    printf(" variogram table: %s\n", fname);
    free(sx);
    free(sy);
    free(sz);
    free(nlag);
    free(gam);
}

/* ------------------------------------------------------------------ conditioning reader, f90:729-855 */

static void condition_field(double *res, const int n[3], int nreal, const double xmin[3], const double d[3],
                            const ora_struct *st, int nst, double nugget, const char *cfile, const char *outbase,
                            recfile *unit)
{
    double t0 = now_s();
    recfile own;
    recfile *iu = unit;
    if (!iu) {
        if (rec_open(&own, cfile, 512)) {
            printf(" Conditioning parameter file not found: %s\n", cfile);
            fstop_code(1);
        }
        iu = &own;
    }
    ora_cond_params cp;
    memset(&cp, 0, sizeof cp);
    const char *line = rec_read_a(iu);
    if (!line) {
        fprintf(stderr, "Fortran runtime error: End of file\n");
        exit(2);
    }
    char datafile[600];
    {
        while (*line == ' ') line++;
        size_t k = 0;
        while (line[k] && line[k] != ' ' && k < sizeof datafile - 1) {
            datafile[k] = line[k];
            k++;
        }
        datafile[k] = 0;
    }
    void *a5[5] = {&cp.ixc, &cp.iyc, &cp.izc, &cp.ivc, &cp.iwc};
    ld_or_die(iu, "iiiii", a5, "conditioning block");
    void *a2[2] = {&cp.tmin, &cp.tmax};
    ld_or_die(iu, "dd", a2, "conditioning block");
    void *b2[2] = {&cp.itrans, &cp.skmean};
    ld_or_die(iu, "id", b2, "conditioning block");
    void *c2[2] = {&cp.zlo, &cp.zhi};
    ld_or_die(iu, "dd", c2, "conditioning block");
    void *d2[2] = {&cp.ltail, &cp.ltpar};
    ld_or_die(iu, "id", d2, "conditioning block");
    void *e2[2] = {&cp.utail, &cp.utpar};
    ld_or_die(iu, "id", e2, "conditioning block");
    void *f3[3] = {&cp.rmax, &cp.rmed, &cp.rvert};
    ld_or_die(iu, "ddd", f3, "conditioning block");
    void *g3[3] = {&cp.sa1, &cp.sa2, &cp.sa3};
    ld_or_die(iu, "ddd", g3, "conditioning block");
    void *h1[1] = {&cp.ndmax};
    ld_or_die(iu, "i", h1, "conditioning block");
    if (!unit) rec_close(&own);
    if (cp.ndmax < 1 || cp.ndmax > 100) fstop_msg("cond: ndmax must be in 1..100");
    if (cp.rmax <= 0 || cp.rmed <= 0 || cp.rvert <= 0) fstop_msg("cond: search radii must be positive");

    /* data file, f90:761-803 */
    recfile df;
    if (rec_open(&df, datafile, 512)) {
        printf(" Data file not found: %s\n", datafile);
        fstop_code(1);
    }
    rec_read_a(&df);
    int nvar = 0;
    void *nv[1] = {&nvar};
    ld_or_die(&df, "i", nv, "data file");
    for (int i = 0; i < nvar; i++) rec_read_a(&df);
    int start = df.pos;
    int nraw = 0;
    for (int q = start; q < df.n; q++) {
        const char *s = df.lines[q];
        size_t L = strlen(s);
        while (L > 0 && (s[L - 1] == ' ' || s[L - 1] == '\t')) L--;
        if (L > 0) nraw++;
    }
    double *rows = malloc(sizeof(double) * (size_t)(nraw > 0 ? nraw : 1) * (nvar > 0 ? nvar : 1));
    int nrows = 0;
    int pos = start;
    char kinds[256];
    for (int i = 0; i < nvar && i < 255; i++) kinds[i] = 'd';
    kinds[nvar < 255 ? nvar : 255] = 0;
    for (int i = 1; i <= nraw; i++) {
        if (pos >= df.n) break;
        const char *s = df.lines[pos++];
        size_t L = strlen(s);
        while (L > 0 && (s[L - 1] == ' ' || s[L - 1] == '\t')) L--;
        if (L == 0) continue;
        recfile one;
        char *tmp = strdup(s);
        one.lines = &tmp;
        one.n = 1;
        one.pos = 0;
        void **outp = malloc(sizeof(void *) * (nvar > 0 ? nvar : 1));
        for (int v = 0; v < nvar; v++) outp[v] = &rows[(size_t)nrows * nvar + v];
        int rc = ld_read(&one, kinds, outp);
        free(outp);
        free(tmp);
        if (rc != 0) {
            fflush(stdout);
            fprintf(stderr, "Fortran runtime error: bad data row %d\n", i);
            exit(2);
        }
        nrows++;
    }
    rec_close(&df);

    ora_cond_stats cs;
    double *vrt = malloc(sizeof(double) * (nrows + 1)), *gtt = malloc(sizeof(double) * (nrows + 1));
    double *dxs = malloc(sizeof(double) * (nrows + 1)), *dys = malloc(sizeof(double) * (nrows + 1));
    double *dzs = malloc(sizeof(double) * (nrows + 1)), *dval = malloc(sizeof(double) * (nrows + 1));
    double *dg = malloc(sizeof(double) * (nrows + 1));
    /* the reference prints the data/nscore lines before kriging; the oracle
     * computes everything first and prints the same lines in the same order */
    int rc = ora_condition(res, n, nreal, xmin, d, st, nst, nugget, &cp, rows, nrows, nvar, &cs, vrt, gtt, dxs, dys,
                           dzs, dval, dg);
    free(rows);
    if (rc == 3) fstop_msg("cond: no conditioning data inside the grid");
    int nd = cs.nd;
    printf(" conditioning data: %s nodes used (%s merged, %s outside the grid)\n", II(nd, 8), II(cs.nmerged, 8),
           II(cs.nout, 8));
    char fname[1200];
    if (cp.itrans == 1) {
        snprintf(fname, sizeof fname, "%s_nscore.trn", outbase);
        FILE *fp = fopen(fname, "w");
        fprintf(fp, "SPECSIM3D normal score transform table (value, normal score)\n2\nvalue\nnscore\n");
        for (int i = 0; i < nd; i++) fprintf(fp, "%s%s\n", ES(vrt[i], 17, 8), ES(gtt[i], 17, 8));
        fclose(fp);
        double s = 0.0;
        for (int i = 0; i < nd; i++) s = s + dg[i];
        double mean = s / nd, v = 0.0;
        for (int i = 0; i < nd; i++) v = v + (dg[i] - s / nd) * (dg[i] - s / nd);
        printf(" normal score transform: data mean=%s  variance=%s\n", FF(mean, 9, 4), FF(v / nd, 9, 4));
    }
    snprintf(fname, sizeof fname, "%s_conddata.dat", outbase);
    FILE *fp = fopen(fname, "w");
    fprintf(fp, "SPECSIM3D conditioning data used (grid nodes)\n5\nx\ny\nz\nvalue\ngauss\n");
    for (int i = 0; i < nd; i++)
        fprintf(fp, "%s%s%s%s%s\n", ES(dxs[i], 17, 8), ES(dys[i], 17, 8), ES(dzs[i], 17, 8), ES(dval[i], 17, 8),
                ES(dg[i], 17, 8));
    fclose(fp);
    printf(" super blocks:%s%s%s  (search %d nearest data)\n", II(cs.nsb[0], 5), II(cs.nsb[1], 5), II(cs.nsb[2], 5),
           cp.ndmax);
    double t1 = now_s();
    printf(" mean neighbours per node: %s  (nodes without data: %d, data nodes: %d)\n",
           FF((double)cs.nsum / ((double)n[0] * n[1] * n[2]), 6, 1), cs.nnone, cs.nexact);
    if (cs.nfail > 0) printf(" WARNING: kriging systems regularized: %d\n", cs.nfail);
    char tb[64];
    f_f(tb, 0.0, 10, 2);
    char *tbs = tb;
    while (*tbs == ' ') tbs++;
    printf(" time conditioning: %s s (kriging) + %s s (back transform)\n", FF(t1 - t0, 8, 2), tbs);
    free(vrt);
    free(gtt);
    free(dxs);
    free(dys);
    free(dzs);
    free(dval);
    free(dg);
}

/* ------------------------------------------------------------------ main program, f90:1085-1418 */

int ora_main(int argc, char **argv)
{
    double t0 = now_s();
    char parfile[512] = "SPECSIM3D.PAR";
    if (argc >= 2) snprintf(parfile, sizeof parfile, "%s", argv[1]);
    int binout = 0, vtkall = 0, dovario = 0, docond = 0, ncli = 0, igauss = 0;
    char varfile[512] = "", condfile[512] = "";
    for (int iarg = 2; iarg < argc; iarg++) {
        const char *a = argv[iarg];
        if (!strcmp(a, "--gauss"))
            igauss = 1;
        else if (!strcmp(a, "--bin")) {
            binout = 1;
            ncli++;
        } else if (!strcmp(a, "--vtk")) {
            vtkall = 1;
            ncli++;
        } else if (!strcmp(a, "--vario")) {
            if (++iarg >= argc) fstop_msg("--vario needs a variogram parameter file");
            snprintf(varfile, sizeof varfile, "%s", argv[iarg]);
            dovario = 1;
        } else if (!strcmp(a, "--cond")) {
            if (++iarg >= argc) fstop_msg("--cond needs a conditioning parameter file");
            snprintf(condfile, sizeof condfile, "%s", argv[iarg]);
            docond = 1;
            ncli++;
        } else {
            printf(" unknown option: %s\n", a);
            fstop_code(1);
        }
    }
    recfile pf;
    if (rec_open(&pf, parfile, 256)) {
        printf(" Parameter file not found: %s\n", parfile);
        fstop_code(1);
    }
    /* optional header, f90:1147-1160 */
    int hdrfound = 0;
    for (int ihdr = 1; ihdr <= 30; ihdr++) {
        const char *h = rec_read_a(&pf);
        if (!h) break;
        char up[300];
        size_t L = strlen(h);
        for (size_t q = 0; q <= L; q++) up[q] = (h[q] >= 'a' && h[q] <= 'z') ? (char)(h[q] - 32) : h[q];
        if (strstr(up, "START OF PARAMETERS")) {
            hdrfound = 1;
            break;
        }
    }
    if (!hdrfound) pf.pos = 0;
    double xmin[3], d[3], nugget;
    int n[3], nst;
    void *p3[3] = {&xmin[0], &xmin[1], &xmin[2]};
    ld_or_die(&pf, "ddd", p3, "parameter file");
    void *q3[3] = {&d[0], &d[1], &d[2]};
    ld_or_die(&pf, "ddd", q3, "parameter file");
    void *r3[3] = {&n[0], &n[1], &n[2]};
    ld_or_die(&pf, "iii", r3, "parameter file");
    void *s2[2] = {&nugget, &nst};
    ld_or_die(&pf, "di", s2, "parameter file");
    if (nst < 1 || nst > ORA_MAXST) fstop_msg("nstruct out of range");
    ora_struct st[ORA_MAXST];
    memset(st, 0, sizeof st);
    for (int s = 0; s < nst; s++) {
        void *o8[8] = {&st[s].itype, &st[s].sill, &st[s].ahmax, &st[s].ahmin,
                       &st[s].avert, &st[s].az,   &st[s].dip,   &st[s].plg};
        ld_or_die(&pf, "iddddddd", o8, "parameter file");
        if (st[s].ahmax <= 0 || st[s].ahmin <= 0 || st[s].avert <= 0) fstop_msg("ranges must be positive");
        ora_setrot(&st[s]);
    }
    int iseed = 0, nreal = 0, ipad = 0;
    {
        const char *hl = rec_read_a(&pf);
        if (!hl) {
            fprintf(stderr, "Fortran runtime error: End of file\n");
            exit(2);
        }
        char *tmp = strdup(hl);
        recfile one = {&tmp, 1, 0};
        int ic = 0;
        void *o4[4] = {&iseed, &nreal, &ipad, &ic};
        int ios = ld_read(&one, "iiii", o4);
        if (ios == 0) {
            if (ic == 1) igauss = 1;
            if (ic < 0 || ic > 1) {
                printf(" parameter file: igauss must be 0 or 1\n");
                fstop_code(1);
            }
        } else {
            one.pos = 0;
            void *o3[3] = {&iseed, &nreal, &ipad};
            ld_or_die(&one, "iii", o3, "seed line");
        }
        free(tmp);
    }
    char outbase[300];
    {
        const char *b = rec_read_a(&pf);
        if (!b) {
            fprintf(stderr, "Fortran runtime error: End of file\n");
            exit(2);
        }
        trim_copy(outbase, b, sizeof outbase);
    }
    int outgs = 0, outvtk1a = 0, outvtk1b = 0, outvti = 0, nout = 0, legacy = 0, icond = 0;
    {
        void *o1[1] = {&nout};
        int ios = ld_read(&pf, "i", o1);
        if (ios < 0)
            legacy = 1;
        else if (ios > 0) {
            printf(" parameter file: cannot read the number of outputs (nout)\n");
            fstop_code(1);
        }
    }
    if (!legacy) {
        binout = vtkall = docond = 0;
        if (nout < 1 || nout > 9) {
            printf(" parameter file: nout must be in 1..9\n");
            fstop_code(1);
        }
        for (int io = 1; io <= nout; io++) {
            int icode = 0;
            void *o1[1] = {&icode};
            if (ld_read(&pf, "i", o1) != 0) {
                printf(" parameter file: missing output code\n");
                fstop_code(1);
            }
            if (icode == 1)
                outgs = 1;
            else if (icode == 2)
                vtkall = 1;
            else if (icode == 3)
                binout = 1;
            else if (icode == 4)
                outvti = 1;
            else {
                printf(" parameter file: output code must be 1 (GSLIB), 2 (VTK), 3 (binary) or 4 (VTI)\n");
                fstop_code(1);
            }
        }
        void *o1[1] = {&icond};
        if (ld_read(&pf, "i", o1) != 0) {
            printf(" parameter file: missing conditioning flag (icond)\n");
            fstop_code(1);
        }
        if (icond < 0 || icond > 1) {
            printf(" parameter file: icond must be 0 or 1\n");
            fstop_code(1);
        }
        docond = icond == 1;
        if (ncli > 0) printf(" Note: --bin, --vtk and --cond are ignored: outputs and conditioning are set in the parameter file\n");
    } else {
        if (vtkall) {
        } else if (binout) {
            outvtk1b = 1;
        } else {
            outgs = 1;
            outvtk1a = 1;
        }
    }
    int np[3];
    if (ora_periodic_grid(st, nst, d, n, ipad, np)) fstop_msg("periodic grid too large (>2^27 nodes)");
    printf(" SPECSIM3D  grid:%s%s%s   periodic grid:%s%s%s\n", II(n[0], 6), II(n[1], 6), II(n[2], 6), II(np[0], 6),
           II(np[1], 6), II(np[2], 6));
    size_t ntot = (size_t)np[0] * np[1] * np[2];
    double *amp = malloc(sizeof(double) * ntot);
    ora_spec_stats ss;
    ora_spectrum(st, nst, nugget, d, np, amp, &ss);
    printf(" max |Im S| / max |Re S|        : %s\n", ES(ss.maximag / ss.maxreal, 10, 3));
    printf(" target variance C(0)           : %s\n", FF(ss.c0, 10, 5));
    printf(" sum of positive spectrum       : %s\n", FF(ss.spos, 10, 5));
    printf(" negative spectral mass / total : %s\n", ES(fabs(ss.sneg) / (ss.spos - ss.sneg), 10, 3));
    if (igauss == 1)
        printf(" spectral coefficients : Gaussian (exactly Gaussian field)\n");
    else
        printf(" spectral coefficients : fixed amplitudes, random phases (default)\n");
    double tsp = now_s();
    printf(" time covariance+spectrum: %s s\n", FF(tsp - t0, 8, 2));
    size_t m = (size_t)n[0] * n[1] * n[2];
    double *res = malloc(sizeof(double) * m * (nreal > 0 ? nreal : 1));
    double *zs = malloc(sizeof(double) * 3 * (nreal > 0 ? nreal : 1));
    ora_realize(amp, np, n, iseed, nreal, igauss, res, zs);
    for (int r = 0; r < nreal; r++)
        printf(" realization%s  mean=%s  variance=%s  max|Im|=%s\n", II(r + 1, 3), FF(zs[3 * r], 9, 4),
               FF(zs[3 * r + 1], 9, 4), ES(zs[3 * r + 2], 9, 2));
    free(amp);
    free(zs);
    if (docond) condition_field(res, n, nreal, xmin, d, st, nst, nugget, condfile, outbase, legacy ? NULL : &pf);
    rec_close(&pf);
    double tsm = now_s();
    printf(" time realizations         : %s s\n", FF(tsm - tsp, 8, 2));
    if (dovario) {
        vario_report(varfile, outbase, res, n, nreal, d, st, nst, nugget);
        double tsv = now_s();
        printf(" time variograms           : %s s\n", FF(tsv - tsm, 8, 2));
    }
    char fname[1200];
    if (binout || vtkall || outvtk1b) {
        float *sp = malloc(sizeof(float) * m);
        FILE *fb = NULL;
        if (binout) {
            snprintf(fname, sizeof fname, "%s.bin", outbase);
            fb = fopen(fname, "wb");
        }
        for (int r = 0; r < nreal; r++) {
            for (size_t q = 0; q < m; q++) sp[q] = (float)res[q + m * r];
            if (fb) fwrite(sp, sizeof(float), m, fb);
            if (vtkall || (outvtk1b && r == 0)) {
                snprintf(fname, sizeof fname, "%s_%d.vtk", outbase, r + 1);
                write_vtk_bin(fname, sp, n[0], n[1], n[2], xmin[0], xmin[1], xmin[2], d[0], d[1], d[2],
                              "SPECSIM3D realization");
            }
        }
        if (fb) fclose(fb);
        free(sp);
    }
    if (outvti) {
        snprintf(fname, sizeof fname, "%s.vti", outbase);
        write_vti(fname, res, n[0], n[1], n[2], nreal, xmin[0], xmin[1], xmin[2], d[0], d[1], d[2]);
    }
    if (outgs) {
        snprintf(fname, sizeof fname, "%s.out", outbase);
        FILE *fp = fopen(fname, "w");
        fprintf(fp, "SPECSIM3D realizations\n%s\n", II(nreal, 4));
        for (int r = 1; r <= nreal; r++) fprintf(fp, "sim%d\n", r);
        for (size_t q = 0; q < m; q++) {
            for (int r = 0; r < nreal; r++) fputs(ES(res[q + m * r], 15, 7), fp);
            fputc('\n', fp);
        }
        fclose(fp);
    }
    if (outvtk1a) {
        snprintf(fname, sizeof fname, "%s_1.vtk", outbase);
        FILE *fp = fopen(fname, "w");
        fprintf(fp, "# vtk DataFile Version 3.0\nSPECSIM3D realization 1\nASCII\nDATASET STRUCTURED_POINTS\n");
        fprintf(fp, "DIMENSIONS%s%s%s\n", II(n[0], 6), II(n[1], 6), II(n[2], 6));
        fprintf(fp, "ORIGIN%s%s%s\n", ES(xmin[0], 15, 7), ES(xmin[1], 15, 7), ES(xmin[2], 15, 7));
        fprintf(fp, "SPACING%s%s%s\n", ES(d[0], 15, 7), ES(d[1], 15, 7), ES(d[2], 15, 7));
        fprintf(fp, "POINT_DATA %d\n", n[0] * n[1] * n[2]);
        fprintf(fp, "SCALARS sim float 1\nLOOKUP_TABLE default\n");
        for (int k = 0; k < n[2]; k++)
            for (int j = 0; j < n[1]; j++) {
                for (int i = 0; i < n[0]; i++)
                    fputs(ES(res[i + (size_t)n[0] * (j + (size_t)n[1] * k)], 13, 5), fp);
                fputc('\n', fp);
            }
        fclose(fp);
    }
    free(res);
    double t1 = now_s();
    printf(" elapsed time: %s s\n", FF(t1 - t0, 8, 2));
    return 0;
}

#ifdef ORACLE_MAIN
int main(int argc, char **argv) { return ora_main(argc, argv); }
#endif
