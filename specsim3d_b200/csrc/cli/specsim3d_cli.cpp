// specsim3d_cli.cpp -- drop-in command line of the B200 implementation:
//
//     specsim3d file.par [--vario variofile.par] [--gauss] [--bin] [--vtk] [--cond condfile]
//                        [--precision fp64|fp32]
//
// Reads the reference's parameter-file grammar (src/specsim3d.f90:40-59,
// 1111-1232, conditioning block 740-753), runs the spectral simulation through
// the C ABI of libspecsim3d_gpu.so, and writes the same files and stdout lines
// (f90:307-391, 487-529, 835-855, 1254-1417).  --precision is an added knob
// (default fp64, the reference's arithmetic); it is a command-line flag so the
// parameter-file grammar stays unchanged.
//
// Fortran semantics kept on purpose: list-directed reads continue over lines
// and ignore text after the values; `stop 'text'` ends with status 0 and
// `stop 1` with status 1 (gfortran behaviour).
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/specsim3d_gpu.h"

namespace {

// ---------------------------------------------------------------- Fortran edit descriptors
std::string justify(const std::string& s, int w) {
  if (w <= 0) return s;
  if ((int)s.size() > w) return std::string(w, '*');
  return std::string(w - s.size(), ' ') + s;
}

bool special(double x, int w, std::string& out) {
  if (std::isnan(x)) {
    out = justify("NaN", w);
    return true;
  }
  if (std::isinf(x)) {
    out = justify(x < 0 ? (w >= 9 ? "-Infinity" : "-Inf") : (w >= 8 ? "Infinity" : "Inf"), w);
    return true;
  }
  return false;
}

// ESw.d: one digit before the point, exponent E+dd (or +ddd past 99)
std::string ES(double x, int w, int d) {
  std::string o;
  if (special(x, w, o)) return o;
  char b[80];
  snprintf(b, sizeof b, "%.*E", d, x);
  char* e = strchr(b, 'E');
  int ex = atoi(e + 1);
  *e = 0;
  if (x == 0.0) ex = 0;
  char r[96];
  if (std::abs(ex) <= 99)
    snprintf(r, sizeof r, "%sE%c%02d", b, ex < 0 ? '-' : '+', std::abs(ex));
  else
    snprintf(r, sizeof r, "%s%c%03d", b, ex < 0 ? '-' : '+', std::abs(ex));
  return justify(r, w);
}

// Fw.d (the leading zero is dropped when the field is otherwise too narrow)
std::string F(double x, int w, int d) {
  std::string o;
  if (special(x, w, o)) return o;
  char b[400];
  snprintf(b, sizeof b, "%.*f", d, x);
  std::string s = b;
  if ((int)s.size() > w) {
    if (s.rfind("0.", 0) == 0) s.erase(0, 1);
    else if (s.rfind("-0.", 0) == 0) s.erase(1, 1);
  }
  return justify(s, w);
}

std::string I(long long v, int w) { return justify(std::to_string(v), w); }

[[noreturn]] void stop_code(int code) {
  fflush(stdout);
  fprintf(stderr, "STOP %d\n", code);
  exit(code);
}
[[noreturn]] void stop_text(const char* msg) {
  fflush(stdout);
  fprintf(stderr, "STOP %s\n", msg);
  exit(0);
}
[[noreturn]] void runtime_error(const std::string& what) {
  fflush(stdout);
  fprintf(stderr, "Fortran runtime error: %s\n", what.c_str());
  exit(2);
}

// ---------------------------------------------------------------- records and list-directed input
struct Records {
  std::vector<std::string> lines;
  size_t pos = 0;
  bool open(const std::string& path, size_t maxlen) {
    std::ifstream in(path);
    if (!in) return false;
    std::string l;
    while (std::getline(in, l)) {
      while (!l.empty() && (l.back() == '\r' || l.back() == '\n')) l.pop_back();
      if (maxlen && l.size() > maxlen) l.resize(maxlen);
      lines.push_back(l);
    }
    return true;
  }
  const std::string* next() { return pos < lines.size() ? &lines[pos++] : nullptr; }
};

bool is_int(const std::string& t, long long& v) {
  size_t i = 0;
  if (i < t.size() && (t[i] == '+' || t[i] == '-')) i++;
  if (i >= t.size()) return false;
  for (size_t k = i; k < t.size(); k++)
    if (!isdigit((unsigned char)t[k])) return false;
  v = strtoll(t.c_str(), nullptr, 10);
  return true;
}

bool is_real(const std::string& t0, double& v) {
  std::string t = t0;
  for (char& c : t)
    if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'e';
  size_t i = 0, digits = 0;
  if (i < t.size() && (t[i] == '+' || t[i] == '-')) i++;
  while (i < t.size() && isdigit((unsigned char)t[i])) i++, digits++;
  if (i < t.size() && t[i] == '.') {
    i++;
    while (i < t.size() && isdigit((unsigned char)t[i])) i++, digits++;
  }
  if (!digits) {
    char* end = nullptr;
    double x = strtod(t.c_str(), &end);
    if (end && *end == 0 && end != t.c_str() && (std::isinf(x) || std::isnan(x))) {
      v = x;
      return true;
    }
    return false;
  }
  if (i < t.size() && (t[i] == 'e' || t[i] == 'E')) {
    i++;
    if (i < t.size() && (t[i] == '+' || t[i] == '-')) i++;
    size_t e0 = i;
    while (i < t.size() && isdigit((unsigned char)t[i])) i++;
    if (i == e0) return false;
  }
  if (i != t.size()) return false;
  v = strtod(t.c_str(), nullptr);
  return true;
}

// One list-directed READ of items of kinds 'i' or 'd' from successive records.
// 0 ok, -1 end of file, 1 conversion error.  Values are written only when read.
struct Item {
  char kind;
  void* p;
};
int list_read(Records& f, std::vector<Item> items) {
  size_t item = 0, rec = f.pos;
  while (item < items.size()) {
    if (rec >= f.lines.size()) return -1;
    const std::string& s = f.lines[rec];
    size_t i = 0;
    bool prev_comma = false;
    while (item < items.size()) {
      while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) i++;
      if (i >= s.size()) break;
      if (s[i] == '/') {
        f.pos = rec + 1;
        return 0;
      }
      if (s[i] == ',') {
        if (prev_comma) item++;
        prev_comma = true;
        i++;
        continue;
      }
      size_t j = i;
      while (j < s.size() && s[j] != ' ' && s[j] != '\t' && s[j] != ',' && s[j] != '/') j++;
      std::string tok = s.substr(i, j - i);
      i = j;
      prev_comma = false;
      int rep = 1;
      std::string val = tok;
      size_t star = tok.find('*');
      if (star != std::string::npos) {
        long long r;
        if (!is_int(tok.substr(0, star), r) || r < 1) return 1;
        rep = (int)r;
        val = tok.substr(star + 1);
      }
      for (int k = 0; k < rep && item < items.size(); k++, item++) {
        if (val.empty()) continue;
        if (items[item].kind == 'i') {
          long long v;
          if (!is_int(val, v)) return 1;
          *(int*)items[item].p = (int)v;
        } else {
          double v;
          if (!is_real(val, v)) return 1;
          *(double*)items[item].p = v;
        }
      }
      while (i < s.size() && (s[i] == ' ' || s[i] == '\t')) i++;
      if (i < s.size() && s[i] == ',') {
        i++;
        prev_comma = true;
      }
    }
    rec++;
  }
  f.pos = rec;
  return 0;
}

void read_or_die(Records& f, std::vector<Item> items, const char* what) {
  int rc = list_read(f, items);
  if (rc) runtime_error(std::string(rc < 0 ? "End of file" : "Bad value") + " while reading " + what);
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t"), b = s.find_last_not_of(" \t");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void check(int rc, const char* what) {
  if (rc != SS3D_OK) {
    fflush(stdout);
    fprintf(stderr, "specsim3d: %s failed: %s\n", what, ss3d_last_error());
    exit(3);
  }
}

// ---------------------------------------------------------------- writers
void put_be32(FILE* fp, float v) {
  unsigned char b[4], o[4];
  memcpy(b, &v, 4);
  o[0] = b[3];
  o[1] = b[2];
  o[2] = b[1];
  o[3] = b[0];
  fwrite(o, 1, 4, fp);
}

// legacy VTK, binary big-endian float32 STRUCTURED_POINTS (f90:362-391)
void write_vtk_bin(const std::string& fname, const float* a, const int n[3], const double x0[3], const double d[3],
                   const char* title) {
  FILE* fp = fopen(fname.c_str(), "wb");
  if (!fp) return;
  fprintf(fp, "# vtk DataFile Version 3.0\n%s\nBINARY\nDATASET STRUCTURED_POINTS\n", title);
  fprintf(fp, "DIMENSIONS %d %d %d\n", n[0], n[1], n[2]);
  fprintf(fp, "ORIGIN %s %s %s\n", ES(x0[0], 16, 8).c_str(), ES(x0[1], 16, 8).c_str(), ES(x0[2], 16, 8).c_str());
  fprintf(fp, "SPACING %s %s %s\n", ES(d[0], 16, 8).c_str(), ES(d[1], 16, 8).c_str(), ES(d[2], 16, 8).c_str());
  fprintf(fp, "POINT_DATA %lld\nSCALARS sim float 1\nLOOKUP_TABLE default\n", (long long)n[0] * n[1] * n[2]);
  const size_t m = (size_t)n[0] * n[1] * n[2];
  for (size_t q = 0; q < m; q++) put_be32(fp, a[q]);
  fputc('\n', fp);
  fclose(fp);
}

// VTK XML ImageData, raw appended little-endian float32, UInt64 headers
// (f90:307-359), written in three parts so that realizations can be appended
// as they arrive: the header (it depends on the sizes only), one block per
// realization, the footer
FILE* vti_open(const std::string& fname, const int n[3], int nreal, const double x0[3], const double d[3]) {
  const uint16_t probe = 1;
  if (*(const unsigned char*)&probe != 1) stop_text("write_vti: big-endian machines are not supported");
  FILE* fp = fopen(fname.c_str(), "wb");
  if (!fp) return nullptr;
  const long long nbytes = 4LL * n[0] * n[1] * n[2];
  char ext[128];
  snprintf(ext, sizeof ext, "0 %d 0 %d 0 %d", n[0] - 1, n[1] - 1, n[2] - 1);
  fprintf(fp, "<?xml version=\"1.0\"?>\n");
  fprintf(fp, "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n");
  fprintf(fp, "  <ImageData WholeExtent=\"%s\" Origin=\" %s %s %s\" Spacing=\" %s %s %s\">\n", ext,
          ES(x0[0], 16, 8).c_str(), ES(x0[1], 16, 8).c_str(), ES(x0[2], 16, 8).c_str(), ES(d[0], 16, 8).c_str(),
          ES(d[1], 16, 8).c_str(), ES(d[2], 16, 8).c_str());
  fprintf(fp, "    <Piece Extent=\"%s\">\n      <PointData Scalars=\"sim_1\">\n", ext);
  for (int r = 1; r <= nreal; r++)
    fprintf(fp, "        <DataArray type=\"Float32\" Name=\"sim_%d\" format=\"appended\" offset=\"%lld\"/>\n", r,
            (nbytes + 8) * (long long)(r - 1));
  fprintf(fp, "      </PointData>\n      <CellData/>\n    </Piece>\n  </ImageData>\n");
  fprintf(fp, "  <AppendedData encoding=\"raw\">\n   _");
  return fp;
}
void vti_block(FILE* fp, const float* a, size_t m) {
  const uint64_t nb = 4ull * m;
  fwrite(&nb, 8, 1, fp);
  fwrite(a, sizeof(float), m, fp);
}
void vti_close(FILE* fp) {
  fprintf(fp, "\n  </AppendedData>\n</VTKFile>\n");
  fclose(fp);
}

void write_vti(const std::string& fname, const double* res, const int n[3], int nreal, const double x0[3],
               const double d[3]) {
  FILE* fp = vti_open(fname, n, nreal, x0, d);
  if (!fp) return;
  const size_t m = (size_t)n[0] * n[1] * n[2];
  std::vector<float> sp(m);
  for (int r = 0; r < nreal; r++) {
    for (size_t q = 0; q < m; q++) sp[q] = (float)res[q + m * r];
    vti_block(fp, sp.data(), m);
  }
  vti_close(fp);
}

// ---------------------------------------------------------------- variogram report (f90:434-529)
void vario_report(const std::string& varfile, const std::string& outbase, const double* res, const int n[3],
                  int nreal, const double d[3], const std::vector<ss3d_struct>& st, double nugget) {
  Records vf;
  if (!vf.open(varfile, 0)) {
    printf(" cannot open variogram file: %s\n", varfile.c_str());
    return;
  }
  int ndir = 0, iper = 0;
  read_or_die(vf, {{'i', &ndir}, {'i', &iper}}, "variogram file");
  std::vector<int> sx(ndir), sy(ndir), sz(ndir), nlag(ndir);
  for (int k = 0; k < ndir; k++)
    read_or_die(vf, {{'i', &sx[k]}, {'i', &sy[k]}, {'i', &sz[k]}, {'i', &nlag[k]}}, "variogram file");
  int nlagmax = 0;
  for (int k = 0; k < ndir; k++) nlagmax = std::max(nlagmax, nlag[k]);
  std::vector<double> gam((size_t)std::max(1, nlagmax) * std::max(1, ndir) * std::max(1, nreal), 0.0);
  std::vector<int64_t> np((size_t)std::max(1, nlagmax) * std::max(1, ndir), 0);
  check(ss3d_vario(res, n, nreal, ndir, sx.data(), sy.data(), sz.data(), nlag.data(), gam.data(), np.data()),
        "ss3d_vario");
  double c0 = nugget;
  for (const auto& s : st) c0 = c0 + s.sill;
  const std::string fname = outbase + "_vario.csv";
  FILE* fp = fopen(fname.c_str(), "w");
  fprintf(fp, "dir,sx,sy,sz,lag,h,npairs,gamma_model,gamma_mean,gamma_sd");
  if (iper == 1)
    for (int r = 1; r <= nreal; r++) fprintf(fp, ",gamma_r%d", r);
  fprintf(fp, "\n");
  printf(" variograms (Fortran): direction  lags  RMS(mean-model)  max|err|   [rising part, gamma_model < 0.95 sill]\n");
  const size_t gs = (size_t)nlagmax * ndir;
  for (int k = 0; k < ndir; k++) {
    double rms = 0.0, mx = 0.0;
    int nfit = 0;
    for (int il = 1; il <= nlag[k]; il++) {
      const int64_t npv = np[(il - 1) + (size_t)nlagmax * k];
      if (npv == 0) continue;
      const double hx = (double)(il * sx[k]) * d[0], hy = (double)(il * sy[k]) * d[1], hz = (double)(il * sz[k]) * d[2];
      const double h = sqrt(hx * hx + hy * hy + hz * hz);
      double cv = 0.0;
      check(ss3d_covariance(st.data(), (int)st.size(), nugget, hx, hy, hz, &cv), "ss3d_covariance");
      const double gth = c0 - cv;
      const double* g = &gam[(il - 1) + (size_t)nlagmax * k];
      double s = 0.0;
      for (int r = 0; r < nreal; r++) s = s + g[gs * r];
      const double gm = s / (double)nreal;
      double gsd = 0.0;
      if (nreal > 1) {
        double v = 0.0;
        for (int r = 0; r < nreal; r++) v = v + (g[gs * r] - gm) * (g[gs * r] - gm);
        gsd = sqrt(v / (double)(nreal - 1));
      }
      fprintf(fp, "%d,%d,%d,%d,%d,%s,%lld,%s,%s,%s", k + 1, sx[k], sy[k], sz[k], il, ES(h, 14, 6).c_str(),
              (long long)npv, ES(gth, 14, 6).c_str(), ES(gm, 14, 6).c_str(), ES(gsd, 14, 6).c_str());
      if (iper == 1)
        for (int r = 0; r < nreal; r++) fprintf(fp, ",%s", ES(g[gs * r], 14, 6).c_str());
      fprintf(fp, "\n");
      if (gth < 0.95 * c0) {
        const double e = gm - gth;
        rms = rms + e * e;
        mx = std::max(mx, std::fabs(e));
        nfit++;
      }
    }
    if (nfit > 0) rms = sqrt(rms / (double)nfit);
    printf("   dir%s%s%s%s%s%s%s\n", I(k + 1, 3).c_str(), I(sx[k], 4).c_str(), I(sy[k], 4).c_str(), I(sz[k], 4).c_str(),
           I(nlag[k], 6).c_str(), F(rms, 12, 5).c_str(), F(mx, 12, 5).c_str());
  }
  fclose(fp);
  printf(" variogram table: %s\n", fname.c_str());
}

// ---------------------------------------------------------------- conditioning (f90:729-930)
void condition(double* res, const int n[3], int nreal, const double xmin[3], const double d[3],
               const std::vector<ss3d_struct>& st, double nugget, const std::string& cfile, const std::string& outbase,
               Records* unit, int precision) {
  const double t0 = now();
  Records own;
  Records* iu = unit;
  if (!iu) {
    if (!own.open(cfile, 512)) {
      printf(" Conditioning parameter file not found: %s\n", cfile.c_str());
      stop_code(1);
    }
    iu = &own;
  }
  const std::string* line = iu->next();
  if (!line) runtime_error("End of file");
  std::string datafile;
  {
    std::string l = *line;
    size_t a = l.find_first_not_of(' ');
    l = a == std::string::npos ? std::string() : l.substr(a);
    datafile = l.substr(0, l.find(' '));
  }
  ss3d_cond_params cp{};
  read_or_die(*iu, {{'i', &cp.ixc}, {'i', &cp.iyc}, {'i', &cp.izc}, {'i', &cp.ivc}, {'i', &cp.iwc}}, "conditioning block");
  read_or_die(*iu, {{'d', &cp.tmin}, {'d', &cp.tmax}}, "conditioning block");
  read_or_die(*iu, {{'i', &cp.itrans}, {'d', &cp.skmean}}, "conditioning block");
  read_or_die(*iu, {{'d', &cp.zmin}, {'d', &cp.zmax}}, "conditioning block");
  read_or_die(*iu, {{'i', &cp.ltail}, {'d', &cp.ltpar}}, "conditioning block");
  read_or_die(*iu, {{'i', &cp.utail}, {'d', &cp.utpar}}, "conditioning block");
  read_or_die(*iu, {{'d', &cp.radius[0]}, {'d', &cp.radius[1]}, {'d', &cp.radius[2]}}, "conditioning block");
  read_or_die(*iu, {{'d', &cp.angles[0]}, {'d', &cp.angles[1]}, {'d', &cp.angles[2]}}, "conditioning block");
  read_or_die(*iu, {{'i', &cp.ndmax}}, "conditioning block");
  if (cp.ndmax < 1 || cp.ndmax > 100) stop_text("cond: ndmax must be in 1..100");
  if (cp.radius[0] <= 0 || cp.radius[1] <= 0 || cp.radius[2] <= 0) stop_text("cond: search radii must be positive");
  // GSLIB data file: title, nvar, nvar names, rows (f90:761-803)
  Records df;
  if (!df.open(datafile, 512)) {
    printf(" Data file not found: %s\n", datafile.c_str());
    stop_code(1);
  }
  df.next();
  int nvar = 0;
  read_or_die(df, {{'i', &nvar}}, "data file");
  for (int q = 0; q < nvar; q++) df.next();
  const size_t start = df.pos;
  int nraw = 0;
  for (size_t q = start; q < df.lines.size(); q++)
    if (!trim(df.lines[q]).empty()) nraw++;
  std::vector<double> rows;
  int nrows = 0;
  size_t pos = start;
  for (int q = 1; q <= nraw; q++) {   // blank lines use up iterations, as in the reference
    if (pos >= df.lines.size()) break;
    const std::string& l = df.lines[pos++];
    if (trim(l).empty()) continue;
    Records one;
    one.lines.push_back(l);
    std::vector<double> row(nvar);
    std::vector<Item> items;
    for (int v = 0; v < nvar; v++) items.push_back({'d', &row[v]});
    if (list_read(one, items)) runtime_error("bad data row " + std::to_string(q));
    rows.insert(rows.end(), row.begin(), row.end());
    nrows++;
  }
  ss3d_cond_stats cs{};
  std::vector<double> vrt(nrows + 1), gtt(nrows + 1), dxs(nrows + 1), dys(nrows + 1), dzs(nrows + 1),
      dval(nrows + 1), dg(nrows + 1);
  const int rc = ss3d_condition(res, n, nreal, xmin, d, st.data(), (int)st.size(), nugget, &cp, rows.data(), nrows,
                                nvar, precision, &cs, vrt.data(), gtt.data(), dxs.data(), dys.data(), dzs.data(),
                                dval.data(), dg.data());
  if (rc == SS3D_ENODATA) stop_text("cond: no conditioning data inside the grid");
  check(rc, "ss3d_condition");
  printf(" conditioning data: %s nodes used (%s merged, %s outside the grid)\n", I(cs.nd, 8).c_str(),
         I(cs.nmerged, 8).c_str(), I(cs.nout, 8).c_str());
  if (cp.itrans == 1) {
    FILE* fp = fopen((outbase + "_nscore.trn").c_str(), "w");
    fprintf(fp, "SPECSIM3D normal score transform table (value, normal score)\n2\nvalue\nnscore\n");
    for (int q = 0; q < cs.nd; q++) fprintf(fp, "%s%s\n", ES(vrt[q], 17, 8).c_str(), ES(gtt[q], 17, 8).c_str());
    fclose(fp);
    printf(" normal score transform: data mean=%s  variance=%s\n", F(cs.data_mean, 9, 4).c_str(),
           F(cs.data_var, 9, 4).c_str());
  }
  FILE* fp = fopen((outbase + "_conddata.dat").c_str(), "w");
  fprintf(fp, "SPECSIM3D conditioning data used (grid nodes)\n5\nx\ny\nz\nvalue\ngauss\n");
  for (int q = 0; q < cs.nd; q++)
    fprintf(fp, "%s%s%s%s%s\n", ES(dxs[q], 17, 8).c_str(), ES(dys[q], 17, 8).c_str(), ES(dzs[q], 17, 8).c_str(),
            ES(dval[q], 17, 8).c_str(), ES(dg[q], 17, 8).c_str());
  fclose(fp);
  printf(" super blocks:%s%s%s  (search %d nearest data)\n", I(cs.nsb[0], 5).c_str(), I(cs.nsb[1], 5).c_str(),
         I(cs.nsb[2], 5).c_str(), cp.ndmax);
  const double t1 = now();
  printf(" mean neighbours per node: %s  (nodes without data: %d, data nodes: %d)\n",
         F((double)cs.nsum / ((double)n[0] * n[1] * n[2]), 6, 1).c_str(), cs.nnone, cs.nexact);
  if (cs.nfail > 0) printf(" WARNING: kriging systems regularized: %d\n", cs.nfail);
  printf(" time conditioning: %s s (kriging) + %s s (back transform)\n", F(t1 - t0, 8, 2).c_str(),
         trim(F(0.0, 10, 2)).c_str());
}

}  // namespace

int main(int argc, char** argv) {
  const double t0 = now();
  std::string parfile = argc >= 2 ? argv[1] : "SPECSIM3D.PAR";
  bool binout = false, vtkall = false, dovario = false, docond = false;
  int ncli = 0, igauss = 0, precision = SS3D_FP64;
  std::string varfile, condfile;
  for (int a = 2; a < argc; a++) {
    const std::string s = argv[a];
    if (s == "--gauss") {
      igauss = 1;
    } else if (s == "--bin") {
      binout = true;
      ncli++;
    } else if (s == "--vtk") {
      vtkall = true;
      ncli++;
    } else if (s == "--vario") {
      if (++a >= argc) stop_text("--vario needs a variogram parameter file");
      varfile = argv[a];
      dovario = true;
    } else if (s == "--cond") {
      if (++a >= argc) stop_text("--cond needs a conditioning parameter file");
      condfile = argv[a];
      docond = true;
      ncli++;
    } else if (s == "--precision") {
      if (++a >= argc) stop_text("--precision needs fp64 or fp32");
      const std::string p = argv[a];
      if (p == "fp32") precision = SS3D_FP32;
      else if (p == "fp64") precision = SS3D_FP64;
      else stop_text("--precision needs fp64 or fp32");
    } else {
      printf(" unknown option: %s\n", s.c_str());
      stop_code(1);
    }
  }
  Records pf;
  if (!pf.open(parfile, 256)) {
    printf(" Parameter file not found: %s\n", parfile.c_str());
    stop_code(1);
  }
  // optional header up to a line containing START OF PARAMETERS (first 30 lines)
  bool hdr = false;
  for (int q = 0; q < 30; q++) {
    const std::string* h = pf.next();
    if (!h) break;
    std::string up = *h;
    for (char& c : up) c = (char)toupper((unsigned char)c);
    if (up.find("START OF PARAMETERS") != std::string::npos) {
      hdr = true;
      break;
    }
  }
  if (!hdr) pf.pos = 0;
  double xmin[3], d[3], nugget = 0;
  int n[3], nst = 0;
  read_or_die(pf, {{'d', &xmin[0]}, {'d', &xmin[1]}, {'d', &xmin[2]}}, "parameter file");
  read_or_die(pf, {{'d', &d[0]}, {'d', &d[1]}, {'d', &d[2]}}, "parameter file");
  read_or_die(pf, {{'i', &n[0]}, {'i', &n[1]}, {'i', &n[2]}}, "parameter file");
  read_or_die(pf, {{'d', &nugget}, {'i', &nst}}, "parameter file");
  if (nst < 1 || nst > 10) stop_text("nstruct out of range");
  std::vector<ss3d_struct> st(nst);
  for (auto& s : st) {
    read_or_die(pf, {{'i', &s.itype}, {'d', &s.sill}, {'d', &s.ahmax}, {'d', &s.ahmin}, {'d', &s.avert},
                     {'d', &s.azimuth}, {'d', &s.dip}, {'d', &s.plunge}},
                "parameter file");
    if (s.ahmax <= 0 || s.ahmin <= 0 || s.avert <= 0) stop_text("ranges must be positive");
  }
  int iseed = 0, nreal = 0, ipad = 0;
  {
    const std::string* hl = pf.next();
    if (!hl) runtime_error("End of file");
    Records one;
    one.lines.push_back(*hl);
    int ic = 0;
    if (list_read(one, {{'i', &iseed}, {'i', &nreal}, {'i', &ipad}, {'i', &ic}}) == 0) {
      if (ic == 1) igauss = 1;
      if (ic < 0 || ic > 1) {
        printf(" parameter file: igauss must be 0 or 1\n");
        stop_code(1);
      }
    } else {
      one.pos = 0;
      read_or_die(one, {{'i', &iseed}, {'i', &nreal}, {'i', &ipad}}, "seed line");
    }
  }
  std::string outbase;
  {
    const std::string* b = pf.next();
    if (!b) runtime_error("End of file");
    outbase = trim(*b);
  }
  bool outgs = false, outvtk1a = false, outvtk1b = false, outvti = false, legacy = false;
  int nout = 0, icond = 0;
  {
    const int rc = list_read(pf, {{'i', &nout}});
    if (rc < 0) legacy = true;
    else if (rc > 0) {
      printf(" parameter file: cannot read the number of outputs (nout)\n");
      stop_code(1);
    }
  }
  if (!legacy) {
    binout = vtkall = docond = false;
    if (nout < 1 || nout > 9) {
      printf(" parameter file: nout must be in 1..9\n");
      stop_code(1);
    }
    for (int q = 0; q < nout; q++) {
      int code = 0;
      if (list_read(pf, {{'i', &code}}) != 0) {
        printf(" parameter file: missing output code\n");
        stop_code(1);
      }
      if (code == 1) outgs = true;
      else if (code == 2) vtkall = true;
      else if (code == 3) binout = true;
      else if (code == 4) outvti = true;
      else {
        printf(" parameter file: output code must be 1 (GSLIB), 2 (VTK), 3 (binary) or 4 (VTI)\n");
        stop_code(1);
      }
    }
    if (list_read(pf, {{'i', &icond}}) != 0) {
      printf(" parameter file: missing conditioning flag (icond)\n");
      stop_code(1);
    }
    if (icond < 0 || icond > 1) {
      printf(" parameter file: icond must be 0 or 1\n");
      stop_code(1);
    }
    docond = icond == 1;
    if (ncli > 0) printf(" Note: --bin, --vtk and --cond are ignored: outputs and conditioning are set in the parameter file\n");
  } else if (vtkall) {
  } else if (binout) {
    outvtk1b = true;
  } else {
    outgs = outvtk1a = true;
  }
  int np[3];
  int rc = ss3d_grid_size(st.data(), nst, d, n, ipad, np);
  if (rc == SS3D_ETOOLARGE) stop_text("periodic grid too large (>2^27 nodes)");
  check(rc, "ss3d_grid_size");
  printf(" SPECSIM3D  grid:%s%s%s   periodic grid:%s%s%s\n", I(n[0], 6).c_str(), I(n[1], 6).c_str(), I(n[2], 6).c_str(),
         I(np[0], 6).c_str(), I(np[1], 6).c_str(), I(np[2], 6).c_str());
  fflush(stdout);
  ss3d_spectrum* sp = nullptr;
  ss3d_spec_stats ss{};
  check(ss3d_spectrum_create(st.data(), nst, nugget, d, n, ipad, &sp, &ss), "ss3d_spectrum_create");
  printf(" max |Im S| / max |Re S|        : %s\n", ES(ss.maximag / ss.maxreal, 10, 3).c_str());
  printf(" target variance C(0)           : %s\n", F(ss.c0, 10, 5).c_str());
  printf(" sum of positive spectrum       : %s\n", F(ss.spos, 10, 5).c_str());
  printf(" negative spectral mass / total : %s\n", ES(std::fabs(ss.sneg) / (ss.spos - ss.sneg), 10, 3).c_str());
  if (igauss == 1) printf(" spectral coefficients : Gaussian (exactly Gaussian field)\n");
  else printf(" spectral coefficients : fixed amplitudes, random phases (default)\n");
  const double tsp = now();
  printf(" time covariance+spectrum: %s s\n", F(tsp - t0, 8, 2).c_str());
  const size_t m = (size_t)n[0] * n[1] * n[2];
  auto stats_line = [&](int r, const double* z) {
    printf(" realization%s  mean=%s  variance=%s  max|Im|=%s\n", I(r + 1, 3).c_str(), F(z[0], 9, 4).c_str(),
           F(z[1], 9, 4).c_str(), ES(z[2], 9, 2).c_str());
  };
  if (!docond && !dovario && !outgs && !outvtk1a) {
    // Streaming: only float32 files are written (.bin, .vti, binary VTK), and
    // none needs all realizations at once.  Chunks of about 64 MB are
    // realized straight to float32 (the same rounding as the conversion of
    // the FP64 values below) and written by a second thread while the next
    // chunk is computed, instead of holding every realization in memory.
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)std::max(nreal, 1), ((size_t)64 << 20) / (4 * m)));
    std::vector<float> buf[2] = {std::vector<float>(m * chunk), std::vector<float>(m * chunk)};
    std::vector<double> zs(3 * (size_t)chunk);
    FILE* fb = binout ? fopen((outbase + ".bin").c_str(), "wb") : nullptr;
    FILE* fv = outvti ? vti_open(outbase + ".vti", n, nreal, xmin, d) : nullptr;
    std::thread writer;
    for (int r0 = 0, c = 0; r0 < nreal; r0 += chunk, ++c) {
      const int nb = std::min(chunk, nreal - r0);
      std::vector<float>& out = buf[c & 1];
      check(ss3d_realize(sp, iseed, r0, nb, igauss, precision, out.data(), SS3D_OUT_F32, zs.data()), "ss3d_realize");
      for (int r = 0; r < nb; r++) stats_line(r0 + r, &zs[3 * (size_t)r]);
      if (writer.joinable()) writer.join();
      writer = std::thread([&, r0, nb, c] {
        const float* a = buf[c & 1].data();
        if (fb) fwrite(a, sizeof(float), m * nb, fb);
        for (int r = 0; r < nb; r++) {
          if (fv) vti_block(fv, a + m * r, m);
          if (vtkall || (outvtk1b && r0 + r == 0))
            write_vtk_bin(outbase + "_" + std::to_string(r0 + r + 1) + ".vtk", a + m * r, n, xmin, d,
                          "SPECSIM3D realization");
        }
      });
    }
    if (writer.joinable()) writer.join();
    if (fb) fclose(fb);
    if (fv) vti_close(fv);
    ss3d_spectrum_free(sp);
    printf(" time realizations         : %s s\n", F(now() - tsp, 8, 2).c_str());
    printf(" elapsed time: %s s\n", F(now() - t0, 8, 2).c_str());
    return 0;
  }
  std::vector<double> res(m * std::max(nreal, 1));
  std::vector<double> zs(3 * (size_t)std::max(nreal, 1));
  check(ss3d_realize(sp, iseed, 0, nreal, igauss, precision, res.data(), SS3D_OUT_F64, zs.data()), "ss3d_realize");
  ss3d_spectrum_free(sp);
  for (int r = 0; r < nreal; r++) stats_line(r, &zs[3 * (size_t)r]);
  if (docond) condition(res.data(), n, nreal, xmin, d, st, nugget, condfile, outbase, legacy ? nullptr : &pf, precision);
  const double tsm = now();
  printf(" time realizations         : %s s\n", F(tsm - tsp, 8, 2).c_str());
  if (dovario) {
    vario_report(varfile, outbase, res.data(), n, nreal, d, st, nugget);
    printf(" time variograms           : %s s\n", F(now() - tsm, 8, 2).c_str());
  }
  if (binout || vtkall || outvtk1b) {
    std::vector<float> sp32(m);
    FILE* fb = binout ? fopen((outbase + ".bin").c_str(), "wb") : nullptr;
    for (int r = 0; r < nreal; r++) {
      for (size_t q = 0; q < m; q++) sp32[q] = (float)res[q + m * r];
      if (fb) fwrite(sp32.data(), sizeof(float), m, fb);
      if (vtkall || (outvtk1b && r == 0))
        write_vtk_bin(outbase + "_" + std::to_string(r + 1) + ".vtk", sp32.data(), n, xmin, d, "SPECSIM3D realization");
    }
    if (fb) fclose(fb);
  }
  if (outvti) write_vti(outbase + ".vti", res.data(), n, nreal, xmin, d);
  if (outgs) {
    FILE* fp = fopen((outbase + ".out").c_str(), "w");
    fprintf(fp, "SPECSIM3D realizations\n%s\n", I(nreal, 4).c_str());
    for (int r = 1; r <= nreal; r++) fprintf(fp, "sim%d\n", r);
    for (size_t q = 0; q < m; q++) {
      for (int r = 0; r < nreal; r++) fputs(ES(res[q + m * r], 15, 7).c_str(), fp);
      fputc('\n', fp);
    }
    fclose(fp);
  }
  if (outvtk1a) {
    FILE* fp = fopen((outbase + "_1.vtk").c_str(), "w");
    fprintf(fp, "# vtk DataFile Version 3.0\nSPECSIM3D realization 1\nASCII\nDATASET STRUCTURED_POINTS\n");
    fprintf(fp, "DIMENSIONS%s%s%s\n", I(n[0], 6).c_str(), I(n[1], 6).c_str(), I(n[2], 6).c_str());
    fprintf(fp, "ORIGIN%s%s%s\n", ES(xmin[0], 15, 7).c_str(), ES(xmin[1], 15, 7).c_str(), ES(xmin[2], 15, 7).c_str());
    fprintf(fp, "SPACING%s%s%s\n", ES(d[0], 15, 7).c_str(), ES(d[1], 15, 7).c_str(), ES(d[2], 15, 7).c_str());
    fprintf(fp, "POINT_DATA %d\nSCALARS sim float 1\nLOOKUP_TABLE default\n", n[0] * n[1] * n[2]);
    for (int k = 0; k < n[2]; k++)
      for (int j = 0; j < n[1]; j++) {
        for (int i = 0; i < n[0]; i++) fputs(ES(res[i + (size_t)n[0] * (j + (size_t)n[1] * k)], 13, 5).c_str(), fp);
        fputc('\n', fp);
      }
    fclose(fp);
  }
  printf(" elapsed time: %s s\n", F(now() - t0, 8, 2).c_str());
  return 0;
}
