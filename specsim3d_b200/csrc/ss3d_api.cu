// ss3d_api.cu -- host side of the C ABI declared in include/specsim3d_gpu.h:
// model setup (setrot, grid sizing), device context (twiddle and jump-ahead
// tables), spectrum handles, realization batching with host/device output.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/specsim3d_gpu.h"
#include "ss3d_internal.h"

using namespace ss3d;

// ---------------------------------------------------------------- errors and stream
static thread_local std::string g_err;
// stream of the calling host thread (ss3d_set_stream)
static thread_local cudaStream_t g_stream = 0;

static int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

static int cuda_fail(cudaError_t e, const char* what) {
  cudaGetLastError();  // clear a sticky-free error
  return fail(e == cudaErrorMemoryAllocation ? SS3D_ENOMEM : SS3D_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                     \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

extern "C" const char* ss3d_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------- stage profiling
static bool g_prof = false;
static double g_prof_ms[SS3D_NSTAGE];
static int64_t g_prof_launch[SS3D_NSTAGE];
static unsigned long long g_mark_launch[16];

void ss3d::mark(Marks* m, int stage, cudaStream_t st) {
  if (!m || !m->on || m->n >= 16) return;
  if (cudaEventCreate(&m->ev[m->n]) != cudaSuccess) return;
  cudaEventRecord(m->ev[m->n], st);
  m->stage[m->n] = stage;
  g_mark_launch[m->n] = g_launch_count.load();
  m->n++;
}

static void marks_collect(Marks& m) {
  for (int q = 0; q + 1 < m.n; q++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, m.ev[q], m.ev[q + 1]) == cudaSuccess && m.stage[q] >= 0 &&
        m.stage[q] < SS3D_NSTAGE) {
      g_prof_ms[m.stage[q]] += ms;
      g_prof_launch[m.stage[q]] += (int64_t)(g_mark_launch[q + 1] - g_mark_launch[q]);
    }
  }
  for (int q = 0; q < m.n; q++) cudaEventDestroy(m.ev[q]);
  m.n = 0;
}

extern "C" int ss3d_profile(int enable) {
  g_prof = enable != 0;
  for (int q = 0; q < SS3D_NSTAGE; q++) {
    g_prof_ms[q] = 0;
    g_prof_launch[q] = 0;
  }
  return SS3D_OK;
}

extern "C" int ss3d_profile_read(double ms[SS3D_NSTAGE], int64_t launches[SS3D_NSTAGE], int64_t* launches_total) {
  for (int q = 0; q < SS3D_NSTAGE; q++) {
    if (ms) ms[q] = g_prof_ms[q];
    if (launches) launches[q] = g_prof_launch[q];
  }
  if (launches_total) *launches_total = (int64_t)g_launch_count.load();
  return SS3D_OK;
}
extern "C" const char* ss3d_version(void) { return "specsim3d_b200 0.1 (sm_100a)"; }
extern "C" int ss3d_set_stream(void* stream) {
  g_stream = (cudaStream_t)stream;
  return SS3D_OK;
}

// ---------------------------------------------------------------- kernel attributes
cudaError_t ss3d::func_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  size_t& have = done[{dev, kernel}];
  if (bytes <= have) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) have = bytes;
  return e;
}

// ---------------------------------------------------------------- kernel loading
// CUDA loads a kernel when it is first launched (lazy module loading, the
// default), and loading one may synchronise the context: in a serving loop
// the first request that needs a kernel not yet loaded would stall the work
// of every stream behind whatever runs.  ss3d_preload_kernels loads every
// kernel of the library's modules on the current device at once, through the
// driver's module enumeration (entry points fetched at run time).
namespace {
template <typename F> F driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    p = nullptr;
  cudaGetLastError();
  return reinterpret_cast<F>(p);
}
}  // namespace

extern "C" int ss3d_preload_kernels(void) {
  using GetModule = CUresult (*)(CUmodule*, CUfunction);
  using Count = CUresult (*)(unsigned int*, CUmodule);
  using Enumerate = CUresult (*)(CUfunction*, unsigned int, CUmodule);
  using Load = CUresult (*)(CUfunction);
  static const GetModule get_module = driver_fn<GetModule>("cuFuncGetModule");
  static const Count count = driver_fn<Count>("cuModuleGetFunctionCount");
  static const Enumerate enumerate = driver_fn<Enumerate>("cuModuleEnumerateFunctions");
  static const Load load = driver_fn<Load>("cuFuncLoad");
  if (!get_module || !count || !enumerate || !load)
    return fail(SS3D_ECUDA, "the CUDA driver does not offer module enumeration and kernel loading");
  for (const void* anchor : {module_anchor_fft(), module_anchor_cond(), module_anchor_vario(), module_anchor_batch()}) {
    cudaFunction_t f = nullptr;
    CK(cudaGetFuncBySymbol(&f, anchor));
    CUmodule mod = nullptr;
    unsigned int n = 0;
    if (get_module(&mod, reinterpret_cast<CUfunction>(f)) != CUDA_SUCCESS || count(&n, mod) != CUDA_SUCCESS)
      return fail(SS3D_ECUDA, "could not enumerate the kernels of a library module");
    std::vector<CUfunction> fs(n);
    if (n > 0 && enumerate(fs.data(), n, mod) != CUDA_SUCCESS)
      return fail(SS3D_ECUDA, "could not enumerate the kernels of a library module");
    for (CUfunction fn : fs)
      if (load(fn) != CUDA_SUCCESS) return fail(SS3D_ECUDA, "could not load a kernel of the library");
  }
  return SS3D_OK;
}

// ---------------------------------------------------------------- device context
namespace {
struct DevCtx {
  bool ready = false;
  float2* twf = nullptr;
  double2* twd = nullptr;
  uint32_t* ptab = nullptr;
};
std::mutex g_ctx_mu;
DevCtx g_ctx[64];

int get_ctx(DevCtx** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SS3D_EINVAL, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  DevCtx& c = g_ctx[dev];
  if (!c.ready) {
    const int ntw = (1 << (TW_LOG_MAX + 1)) - 1;
    std::vector<float2> hf(ntw);
    std::vector<double2> hd(ntw);
    for (int L = 0; L <= TW_LOG_MAX; ++L) {
      int n = 1 << L;
      for (int m = 0; m < n; ++m) {
        long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
        long double c0 = cosl(ang), s0 = sinl(ang);
        hd[n - 1 + m] = make_double2((double)c0, (double)s0);
        hf[n - 1 + m] = make_float2((float)c0, (float)s0);
      }
    }
    // tab[l*2048 + v] = 16807^(v * 2048^l) mod (2^31 - 1)
    std::vector<uint32_t> ht(3 * 2048);
    uint32_t base = PM_A;
    for (int l = 0; l < 3; ++l) {
      uint32_t acc = 1;
      for (int v = 0; v < 2048; ++v) {
        ht[l * 2048 + v] = acc;
        acc = pm_mulmod(acc, base);
      }
      base = acc;  // base^2048
    }
    CK(cudaMalloc(&c.twf, sizeof(float2) * ntw));
    CK(cudaMalloc(&c.twd, sizeof(double2) * ntw));
    CK(cudaMalloc(&c.ptab, sizeof(uint32_t) * 3 * 2048));
    CK(cudaMemcpy(c.twf, hf.data(), sizeof(float2) * ntw, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.twd, hd.data(), sizeof(double2) * ntw, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.ptab, ht.data(), sizeof(uint32_t) * 3 * 2048, cudaMemcpyHostToDevice));
    // a copy from pageable memory may return before its DMA ends, and the
    // kernels that read the tables can run on non-blocking streams that do not
    // order behind the legacy stream: wait for the copies once, here
    CK(cudaDeviceSynchronize());
    // Spectra, work spaces and temporaries come from the device's
    // stream-ordered pool.  Freed pool memory stays mapped (release threshold
    // unlimited): mapping device pages costs about a millisecond per few MB
    // here, so a spectrum or work space freed by one call and taken again by
    // the next must not be unmapped in between.  ss3d_release_workspace gives
    // the pool's free memory back to the device.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
      uint64_t keep = ~(uint64_t)0;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
    c.ready = true;
  }
  *out = &c;
  return SS3D_OK;
}

}  // namespace

int ss3d::check_ptr(const void* p, int dev, size_t align, const char* what, bool* is_dev) {
  *is_dev = false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return SS3D_OK;   // memory CUDA does not know: ordinary host memory
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) return SS3D_OK;
  *is_dev = true;
  if (a.type == cudaMemoryTypeDevice && a.device != dev)
    return fail(SS3D_EINVAL, "%s is memory of device %d, the work runs on device %d", what, a.device, dev);
  if (align > 1 && ((uintptr_t)p % align) != 0)
    return fail(SS3D_EINVAL, "%s must start on a multiple of %zu bytes (device memory at %p)", what, align, p);
  return SS3D_OK;
}

namespace {

// ---------------------------------------------------------------- model
const double PI = 3.14159265358979323846;  // f90:92

// setrot, f90:107-139 (same expression order as the reference)
void setrot_rc(const ss3d_struct& s, double rot[3][3], double axes[3][3]) {
  double deg = PI / 180.0;
  double alpha = (s.azimuth >= 0.0 && s.azimuth < 270.0) ? (90.0 - s.azimuth) * deg : (450.0 - s.azimuth) * deg;
  double beta = -(s.dip * deg);
  double theta = s.plunge * deg;
  double sina = sin(alpha), cosa = cos(alpha);
  double sinb = sin(beta), cosb = cos(beta);
  double sint = sin(theta), cost = cos(theta);
  double anis1 = s.ahmin / s.ahmax, anis2 = s.avert / s.ahmax;
  double afac1 = 1.0 / fmax(anis1, 1.0e-20), afac2 = 1.0 / fmax(anis2, 1.0e-20);
  rot[0][0] = cosb * cosa;
  rot[0][1] = cosb * sina;
  rot[0][2] = -sinb;
  rot[1][0] = afac1 * (-(cost * sina) + sint * sinb * cosa);
  rot[1][1] = afac1 * (cost * cosa + sint * sinb * sina);
  rot[1][2] = afac1 * (sint * cosb);
  rot[2][0] = afac2 * (sint * sina + cost * sinb * cosa);
  rot[2][1] = afac2 * (-(sint * cosa) + cost * sinb * sina);
  rot[2][2] = afac2 * (cost * cosb);
  for (int c = 0; c < 3; c++) {
    axes[0][c] = rot[0][c] * s.ahmax;
    axes[1][c] = rot[1][c] / afac1 * s.ahmin;
    axes[2][c] = rot[2][c] / afac2 * s.avert;
  }
}

int check_structs(const ss3d_struct* st, int nst) {
  if (!st) return fail(SS3D_EINVAL, "structures pointer is NULL");
  if (nst < 1 || nst > MAXST) return fail(SS3D_EINVAL, "nstruct out of range");
  for (int i = 0; i < nst; i++) {
    if (st[i].ahmax <= 0 || st[i].ahmin <= 0 || st[i].avert <= 0) return fail(SS3D_EINVAL, "ranges must be positive");
    if (st[i].itype < 1 || st[i].itype > 3) {
      // the reference treats any other itype as gaussian (select case default, f90:174)
    }
  }
  return SS3D_OK;
}

void build_model(const ss3d_struct* st, int nst, double nugget, Model& m) {
  memset(&m, 0, sizeof m);
  m.nst = nst;
  m.nugget = nugget;
  for (int i = 0; i < nst; i++) {
    double rot[3][3], axes[3][3];
    setrot_rc(st[i], rot, axes);
    m.itype[i] = st[i].itype;
    m.sill[i] = st[i].sill;
    m.ahmax[i] = st[i].ahmax;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) m.rot[i][3 * r + c] = rot[r][c];
  }
}

int nextpow2(int n) {
  int m = 1;
  while (m < n) m *= 2;
  return m;
}

double cutoff(int itype) { return itype == 1 ? 1.0 : (itype == 2 ? 2.3 : 1.6); }

int grid_size(const ss3d_struct* st, int nst, const double d[3], const int n[3], int ipad, int np[3]) {
  np[0] = nextpow2(n[0]);
  np[1] = nextpow2(n[1]);
  np[2] = nextpow2(n[2]);
  if (ipad == 1) {
    double e[3] = {0, 0, 0};
    for (int s = 0; s < nst; s++) {
      double rot[3][3], axes[3][3];
      setrot_rc(st[s], rot, axes);
      for (int a = 0; a < 3; a++) {
        double ss = axes[0][a] * axes[0][a];
        ss = ss + axes[1][a] * axes[1][a];
        ss = ss + axes[2][a] * axes[2][a];
        e[a] = fmax(e[a], cutoff(st[s].itype) * sqrt(ss) / d[a]);
      }
    }
    int r[3];
    for (int a = 0; a < 3; a++) r[a] = (int)ceil(e[a]);
    np[0] = nextpow2(std::max(n[0] + r[0], 2 * r[0]));
    np[1] = nextpow2(std::max(n[1] + r[1], 2 * r[1]));
    np[2] = n[2] > 1 ? nextpow2(std::max(n[2] + r[2], 2 * r[2])) : 1;
  }
  if ((double)np[0] * (double)np[1] * (double)np[2] > 134217728.0)
    return fail(SS3D_ETOOLARGE, "periodic grid too large (>2^27 nodes)");
  return SS3D_OK;
}

int ilog2i(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}
}  // namespace

extern "C" int ss3d_setrot(const ss3d_struct* s, double rot[9], double axes[9]) {
  if (!s || !rot || !axes) return fail(SS3D_EINVAL, "NULL argument");
  double r[3][3], a[3][3];
  setrot_rc(*s, r, a);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      rot[3 * i + j] = r[i][j];
      axes[3 * i + j] = a[i][j];
    }
  return SS3D_OK;
}

extern "C" int ss3d_covariance(const ss3d_struct* st, int nst, double nugget, double dx, double dy, double dz,
                               double* c) {
  int rc = check_structs(st, nst);
  if (rc) return rc;
  Model m;
  build_model(st, nst, nugget, m);
  *c = covariance(m, dx, dy, dz);
  return SS3D_OK;
}

extern "C" int ss3d_grid_size(const ss3d_struct* st, int nst, const double d[3], const int n[3], int ipad,
                              int np[3]) {
  int rc = check_structs(st, nst);
  if (rc) return rc;
  if (!d || !n || !np) return fail(SS3D_EINVAL, "NULL argument");
  if (n[0] < 1 || n[1] < 1 || n[2] < 1) return fail(SS3D_EINVAL, "grid sizes must be positive");
  return grid_size(st, nst, d, n, ipad, np);
}

// ---------------------------------------------------------------- spectrum handle
struct ss3d_spectrum {
  int dev;
  Geo geo;  // d and D filled per call
  Model model;
  double d[3];
  ss3d_spec_stats stats;
  double* amp64 = nullptr;
  float* amp32 = nullptr;
};

namespace {
int supported_axes(const Geo& g, bool dbl, const char** which) {
  int maxl = dbl ? MAX_LOGN_D : MAX_LOGN_F;
  if (g.npx > 1 && ilog2i(g.npx) - 1 > maxl) { *which = "x"; return 0; }
  if (ilog2i(g.npy) > maxl) { *which = "y"; return 0; }
  if (ilog2i(g.npz) > maxl) { *which = "z"; return 0; }
  return 1;
}

// Work space of the realization path, kept per host thread and device so that
// threads realizing at the same time on their own streams never share it.
// It grows on demand; every call finishes its work before it returns.
struct Workspace {
  void* p = nullptr;
  size_t bytes = 0;
  int dev = 0;
  // stream-ordered release on the thread's stream: no device-wide synchronisation
  void release(cudaStream_t st) {
    if (p) {
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(dev);
      cudaFreeAsync(p, st);
      cudaSetDevice(cur);
    }
    p = nullptr;
    bytes = 0;
  }
  ~Workspace() {
    if (p) {
      cudaSetDevice(dev);
      cudaFree(p);
    }
  }
};
thread_local Workspace g_ws[64];

// Copy stream and events of the host-output path, per host thread and device,
// created on first use and kept (creating them per call costs a few
// microseconds each and serialises with other threads' launches).
struct CopyCtx {
  cudaStream_t cs = nullptr;
  cudaEvent_t done[2] = {nullptr, nullptr};
  cudaEvent_t ready = nullptr;
  int dev = -1;
  ~CopyCtx() {
    if (dev < 0) return;
    cudaSetDevice(dev);
    if (cs) cudaStreamDestroy(cs);
    for (cudaEvent_t ev : {done[0], done[1], ready})
      if (ev) cudaEventDestroy(ev);
  }
};
thread_local CopyCtx g_copy[64];

int copy_ctx(int dev, CopyCtx** out) {
  CopyCtx& c = g_copy[dev];
  if (c.dev < 0) {
    CK(cudaStreamCreateWithFlags(&c.cs, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c.done[0], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.done[1], cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&c.ready, cudaEventDisableTiming));
    c.dev = dev;
  }
  *out = &c;
  return SS3D_OK;
}

int ws_reserve(int dev, size_t bytes, void** ptr) {
  if (dev < 0 || dev >= 64) return fail(SS3D_EINVAL, "device ordinal %d out of range", dev);
  Workspace& w = g_ws[dev];
  if (w.bytes < bytes) {
    w.release(g_stream);
    CK(cudaMallocAsync(&w.p, bytes, g_stream));
    w.bytes = bytes;
    w.dev = dev;
  }
  *ptr = w.p;
  return SS3D_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
}  // namespace

extern "C" int ss3d_spectrum_create(const ss3d_struct* st, int nst, double nugget, const double d[3], const int n[3],
                                    int ipad, ss3d_spectrum** out, ss3d_spec_stats* stats) {
  if (!out) return fail(SS3D_EINVAL, "out is NULL");
  *out = nullptr;
  int rc = check_structs(st, nst);
  if (rc) return rc;
  if (!d || !n) return fail(SS3D_EINVAL, "NULL argument");
  if (n[0] < 1 || n[1] < 1 || n[2] < 1) return fail(SS3D_EINVAL, "grid sizes must be positive");
  int np[3];
  rc = grid_size(st, nst, d, n, ipad, np);
  if (rc) return rc;
  DevCtx* ctx;
  if ((rc = get_ctx(&ctx))) return rc;
  ss3d_spectrum* sp = new ss3d_spectrum();
  CK(cudaGetDevice(&sp->dev));
  Geo& g = sp->geo;
  g.npx = np[0];
  g.npy = np[1];
  g.npz = np[2];
  g.nx = n[0];
  g.ny = n[1];
  g.nz = n[2];
  g.H = np[0] >= 2 ? np[0] / 2 + 1 : 1;
  g.HP = (g.H + 1) & ~1;
  g.d = 1;
  g.D = 0;
  const char* ax = "";
  if (!supported_axes(g, true, &ax)) {
    delete sp;
    return fail(SS3D_ETOOLARGE, "periodic axis %s longer than the supported FP64 transform length", ax);
  }
  memcpy(sp->d, d, sizeof sp->d);
  build_model(st, nst, nugget, sp->model);
  const size_t nh = (size_t)g.npz * g.npy * g.HP;
  cudaStream_t s = g_stream;
  double2* work = nullptr;
  SpecPartial* part = nullptr;
  const int npart = spectrum_parts(g) - 1;
  // temporaries come from the stream-ordered pool: no device-wide synchronisation
  // when they are freed, so that other threads' streams keep running
  cudaError_t e = cudaMallocAsync((void**)&work, sizeof(double2) * nh, s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&sp->amp64, sizeof(double) * nh, s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&sp->amp32, sizeof(float) * nh, s);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&part, sizeof(SpecPartial) * (npart + 1), s);
  if (e == cudaSuccess)
    e = launch_spectrum(sp->model, d, g, work, sp->amp64, sp->amp32, part, npart, part + npart, Tw{ctx->twf, ctx->twd},
                        s);
  SpecPartial res{};
  if (e == cudaSuccess) e = cudaMemcpyAsync(&res, part + npart, sizeof res, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (work) cudaFreeAsync(work, s);
  if (part) cudaFreeAsync(part, s);
  if (e != cudaSuccess) {
    ss3d_spectrum_free(sp);
    return cuda_fail(e, "spectrum");
  }
  sp->stats.np[0] = np[0];
  sp->stats.np[1] = np[1];
  sp->stats.np[2] = np[2];
  sp->stats.c0 = covariance(sp->model, 0.0, 0.0, 0.0);
  sp->stats.maximag = res.maximag;
  sp->stats.maxreal = res.maxreal;
  sp->stats.spos = res.spos;
  sp->stats.sneg = res.sneg;
  if (stats) *stats = sp->stats;
  *out = sp;
  return SS3D_OK;
}

// The amplitudes come from the device's stream-ordered pool and go back to it
// on the calling thread's stream (no device-wide synchronisation); the caller
// has finished every use of the spectrum on other streams.
extern "C" void ss3d_spectrum_free(ss3d_spectrum* sp) {
  if (!sp) return;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(sp->dev);
  if (sp->amp64) cudaFreeAsync(sp->amp64, g_stream);
  if (sp->amp32) cudaFreeAsync(sp->amp32, g_stream);
  cudaSetDevice(cur);
  delete sp;
}

extern "C" int ss3d_spectrum_info(const ss3d_spectrum* sp, int np[3], int n[3], ss3d_spec_stats* stats) {
  if (!sp) return fail(SS3D_EINVAL, "spectrum is NULL");
  if (np) {
    np[0] = sp->geo.npx;
    np[1] = sp->geo.npy;
    np[2] = sp->geo.npz;
  }
  if (n) {
    n[0] = sp->geo.nx;
    n[1] = sp->geo.ny;
    n[2] = sp->geo.nz;
  }
  if (stats) *stats = sp->stats;
  return SS3D_OK;
}

extern "C" int64_t ss3d_spectrum_bytes(const ss3d_spectrum* sp) {
  if (!sp) return 0;
  const size_t nh = (size_t)sp->geo.npz * sp->geo.npy * sp->geo.HP;
  return (int64_t)(nh * (sizeof(double) + sizeof(float)));
}

extern "C" int ss3d_spectrum_amp(const ss3d_spectrum* sp, double* amp) {
  if (!sp || !amp) return fail(SS3D_EINVAL, "NULL argument");
  const Geo& g = sp->geo;
  CK(cudaMemcpy2DAsync(amp, sizeof(double) * g.H, sp->amp64, sizeof(double) * g.HP, sizeof(double) * g.H,
                       (size_t)g.npy * g.npz, cudaMemcpyDeviceToHost, g_stream));
  CK(cudaStreamSynchronize(g_stream));
  return SS3D_OK;
}

// ---------------------------------------------------------------- realizations
namespace {
Geo geo_for_np(Geo g, int igauss) {
  g.d = igauss ? 2 : 1;
  uint64_t N = (uint64_t)g.npx * g.npy * g.npz;
  uint64_t nself = (uint64_t)(g.npx >= 2 ? 2 : 1) * (g.npy >= 2 ? 2 : 1) * (g.npz >= 2 ? 2 : 1);
  g.D = (uint64_t)g.d * ((N + nself) / 2);
  return g;
}
Geo geo_for(const ss3d_spectrum* sp, int igauss) {
  Geo g = sp->geo;
  g.d = igauss ? 2 : 1;
  uint64_t N = (uint64_t)g.npx * g.npy * g.npz;
  uint64_t nself = (uint64_t)(g.npx >= 2 ? 2 : 1) * (g.npy >= 2 ? 2 : 1) * (g.npz >= 2 ? 2 : 1);
  g.D = (uint64_t)g.d * ((N + nself) / 2);
  return g;
}
uint32_t seed0(int iseed) {
  int64_t a = iseed < 0 ? -(int64_t)iseed : (int64_t)iseed;
  return (uint32_t)(a % 2147483646LL + 1);
}
}  // namespace

namespace {
// complex planes per realization in the work space: the first (z) inverse pass
// stores only the planes k < nz that survive the crop
int work_planes(const Geo& g) { return g.npz > 1 ? g.nz : 1; }

// Work-space layout of one realize call: batches of at most 16 realizations
// and about 4 GiB; host output goes through two staging buffers.
struct RealizeLayout {
  int bt;
  size_t per_work, off_work, off_rs, off_apow, off_part, off_zs, off_stage, stage_bytes, total;
};
RealizeLayout realize_layout(const Geo& g, bool dbl, bool dev_out, int nreal, size_t oel) {
  RealizeLayout L{};
  const size_t M = (size_t)g.nx * g.ny * g.nz;
  const size_t cel = dbl ? sizeof(double2) : sizeof(float2);
  L.per_work = (size_t)work_planes(g) * g.npy * g.HP * cel;
  const int nbx = realize_part_blocks(g, dbl);
  const size_t budget = (size_t)4 << 30;
  const size_t per_real = L.per_work + (dev_out ? 0 : 2 * M * oel) + (size_t)g.npy * g.npz * 4 + (size_t)nbx * 16;
  L.bt = (int)std::min<size_t>((size_t)std::max(nreal, 1), std::max<size_t>(1, budget / per_real));
  L.bt = std::min(L.bt, 16);
  if (!dev_out) {
    // host output: chunks of about 32 MB, so that the copy of chunk b to the
    // host (PCIe, several times slower than the kernels) overlaps the kernels
    // of chunk b + 1 instead of waiting for the whole batch
    const size_t chunk = std::max<size_t>(1, ((size_t)32 << 20) / std::max<size_t>(1, M * oel));
    L.bt = (int)std::min<size_t>((size_t)L.bt, chunk);
  }
  L.off_work = 0;
  L.off_rs = align256(L.off_work + L.per_work * L.bt);
  L.off_apow = align256(L.off_rs + (size_t)g.npy * g.npz * 4 * L.bt);
  L.off_part = align256(L.off_apow + (size_t)g.npx * 4);
  L.off_zs = align256(L.off_part + (size_t)nbx * 16 * L.bt);
  L.off_stage = align256(L.off_zs + (size_t)std::max(nreal, 1) * 16);
  L.stage_bytes = dev_out ? 0 : align256(M * oel * L.bt);
  L.total = L.off_stage + 2 * L.stage_bytes;
  return L;
}
}  // namespace

// work-space bytes of a realize call on periodic grid np with output grid n,
// before any spectrum exists (admission control of the serving form); an
// upper bound: host output staged as double
int64_t ss3d::realize_bytes_for(const int np[3], const int n[3], int nreal, int precision, int host_out) {
  Geo g{};
  g.npx = np[0];
  g.npy = np[1];
  g.npz = np[2];
  g.nx = n[0];
  g.ny = n[1];
  g.nz = n[2];
  g.H = np[0] >= 2 ? np[0] / 2 + 1 : 1;
  g.HP = (g.H + 1) & ~1;
  const bool dbl = precision == SS3D_FP64;
  return (int64_t)realize_layout(g, dbl, host_out == 0, nreal, 8).total;
}

extern "C" int64_t ss3d_realize_workspace_bytes(const ss3d_spectrum* sp, int nreal, int precision, int host_out) {
  if (!sp || nreal < 0 || (precision != SS3D_FP64 && precision != SS3D_FP32)) return -1;
  const bool dbl = precision == SS3D_FP64;
  return (int64_t)realize_layout(sp->geo, dbl, host_out == 0, nreal, 8).total;
}

extern "C" int ss3d_release_workspace(void) {
  for (Workspace& w : g_ws) w.release(g_stream);
  cudaStreamSynchronize(g_stream);
  return SS3D_OK;
}

size_t ss3d::pool_premap(size_t bytes) {
  DevCtx* ctx;
  if (get_ctx(&ctx)) return 0;   // also sets the pool's release threshold
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return 0;
  size_t done = 0;
  for (size_t b = bytes; b >= ((size_t)256 << 20) && !done; b /= 2) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, b, st) == cudaSuccess) {
      cudaFreeAsync(p, st);
      done = b;
    }
    cudaGetLastError();
  }
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return done;
}

extern "C" int ss3d_trim_pool(void) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  CK(cudaDeviceGetDefaultMemPool(&pool, dev));
  CK(cudaDeviceSynchronize());
  CK(cudaMemPoolTrimTo(pool, 0));
  return SS3D_OK;
}

extern "C" int ss3d_realize(const ss3d_spectrum* csp, int iseed, int64_t r_first, int nreal, int igauss,
                            int precision, void* out, int out_dtype, double* zstats) {
  ss3d_spectrum* sp = const_cast<ss3d_spectrum*>(csp);
  if (!sp) return fail(SS3D_EINVAL, "spectrum is NULL");
  if (nreal < 0) return fail(SS3D_EINVAL, "nreal must be >= 0");
  if (r_first < 0) return fail(SS3D_EINVAL, "r_first must be >= 0");
  if (igauss != 0 && igauss != 1) return fail(SS3D_EINVAL, "igauss must be 0 or 1");
  if (precision != SS3D_FP64 && precision != SS3D_FP32) return fail(SS3D_EINVAL, "unknown precision %d", precision);
  if (out_dtype != SS3D_OUT_F32 && out_dtype != SS3D_OUT_F64) return fail(SS3D_EINVAL, "unknown out_dtype %d", out_dtype);
  if (nreal == 0) return SS3D_OK;
  if (!out) return fail(SS3D_EINVAL, "out is NULL");
  const bool dbl = precision == SS3D_FP64;
  Geo g = geo_for(sp, igauss);
  const char* ax = "";
  if (!supported_axes(g, dbl, &ax))
    return fail(SS3D_ETOOLARGE, "periodic axis %s longer than the supported transform length", ax);
  // the tables of the spectrum's device: make it current before taking them
  CK(cudaSetDevice(sp->dev));
  DevCtx* ctx;
  int rc;
  if ((rc = get_ctx(&ctx))) return rc;
  cudaStream_t s = g_stream;
  const size_t M = (size_t)g.nx * g.ny * g.nz;
  const size_t oel = out_dtype == SS3D_OUT_F32 ? 4 : 8;
  bool dev_out = false;
  if ((rc = check_ptr(out, sp->dev, (g.nx % 2 == 0 ? 2 : 1) * oel, "out", &dev_out))) return rc;
  const RealizeLayout lay = realize_layout(g, dbl, dev_out, nreal, oel);
  const int bt = lay.bt;
  void* wsp = nullptr;
  if ((rc = ws_reserve(sp->dev, lay.total, &wsp))) return rc;
  char* base = (char*)wsp;
  void* work = base + lay.off_work;
  uint32_t* rs = (uint32_t*)(base + lay.off_rs);
  uint32_t* apow = (uint32_t*)(base + lay.off_apow);
  double* part = (double*)(base + lay.off_part);
  double* zs = (double*)(base + lay.off_zs);
  char* stage[2] = {base + lay.off_stage, base + lay.off_stage + lay.stage_bytes};
  const long long wstride = (long long)work_planes(g) * g.npy * g.HP;
  const uint32_t s0 = seed0(iseed);
  Tw tw{ctx->twf, ctx->twd};
  cudaEvent_t* done = nullptr;
  cudaEvent_t ready = nullptr;
  cudaStream_t cs = nullptr;
  if (!dev_out) {
    CopyCtx* cc = nullptr;
    if ((rc = copy_ctx(sp->dev, &cc))) return rc;
    cs = cc->cs;
    done = cc->done;
    ready = cc->ready;
    // the previous call's copies ended before it returned; order this call's
    // first chunks after them all the same (the events are reused)
    CK(cudaStreamWaitEvent(s, done[0], 0));
    CK(cudaStreamWaitEvent(s, done[1], 0));
  }
  cudaError_t e = cudaSuccess;
  Marks marks;
  marks.on = g_prof;
  const unsigned long long pipes0 = g_pipe_launches.load();
  int ib = 0;
  for (int r0 = 0; r0 < nreal && e == cudaSuccess; r0 += bt, ++ib) {
    int nb = std::min(bt, nreal - r0);
    int slot = ib & 1;
    void* dst = dev_out ? (void*)((char*)out + (size_t)r0 * M * oel) : (void*)stage[slot];
    if (!dev_out && ib >= 2) e = cudaStreamWaitEvent(s, done[slot], 0);
    mark(&marks, 0, s);
    if (e == cudaSuccess) e = launch_rowstates(g, s0, r_first + r0, nb, ctx->ptab, rs, r0 == 0 ? apow : nullptr, s);
    int nblk = 0;
    if (e == cudaSuccess) {
      if (dbl)
        e = launch_realize<double>(g, sp->amp64, rs, apow, (double2*)work, wstride, nb, dst, out_dtype,
                                   zstats ? part : nullptr, &nblk, tw, true, s, &marks);
      else
        e = launch_realize<float>(g, sp->amp32, rs, apow, (float2*)work, wstride, nb, dst, out_dtype,
                                  zstats ? part : nullptr, &nblk, tw, true, s, &marks);
    }
    mark(&marks, 4, s);
    if (e == cudaSuccess && zstats) e = launch_reduce_zstats(part, nblk, nb, zs + 2 * (size_t)r0, s);
    mark(&marks, -1, s);
    if (e == cudaSuccess && !dev_out) {
      e = cudaEventRecord(ready, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, ready, 0);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync((char*)out + (size_t)r0 * M * oel, stage[slot], (size_t)nb * M * oel,
                            cudaMemcpyDeviceToHost, cs);
      if (e == cudaSuccess) e = cudaEventRecord(done[slot], cs);
    }
  }
  std::vector<double> hz;
  if (e == cudaSuccess && zstats) {
    hz.resize(2 * (size_t)nreal);
    e = cudaMemcpyAsync(hz.data(), zs, sizeof(double) * 2 * nreal, cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && cs) e = cudaStreamSynchronize(cs);
  if (marks.on) marks_collect(marks);
  if (e != cudaSuccess) return cuda_fail(e, "realize");
  if (g_pipe_launches.load() != pipes0 && pipe_error_take(s))
    return fail(SS3D_ECUDA, "realize: a bulk-copy wait of the middle pass timed out");
  if (zstats) {
    for (int r = 0; r < nreal; r++) {
      double mean = hz[2 * r] / (double)M;
      zstats[3 * r] = mean;
      zstats[3 * r + 1] = hz[2 * r + 1] / (double)M - mean * mean;
      zstats[3 * r + 2] = 0.0;
    }
  }
  return SS3D_OK;
}

// ---------------------------------------------------------------- full-grid transform (test export)
extern "C" int ss3d_fft3d(double* a, int nx, int ny, int nz, int isign) {
  if (!a) return fail(SS3D_EINVAL, "a is NULL");
  if (isign != -1 && isign != 1) return fail(SS3D_EINVAL, "isign must be -1 or +1");
  auto pow2 = [](int v) { return v >= 1 && (v & (v - 1)) == 0; };
  if (!pow2(nx) || !pow2(ny) || !pow2(nz)) return fail(SS3D_EINVAL, "grid sizes must be powers of two");
  if (ilog2i(nx) > MAX_LOGN_D || ilog2i(ny) > MAX_LOGN_D || ilog2i(nz) > MAX_LOGN_D)
    return fail(SS3D_ETOOLARGE, "axis longer than the supported FP64 transform length (%d)", 1 << MAX_LOGN_D);
  if ((double)nx * ny * nz > 134217728.0) return fail(SS3D_ETOOLARGE, "grid above 2^27 nodes");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  DevCtx* ctx;
  int rc;
  if ((rc = get_ctx(&ctx))) return rc;
  const size_t n = (size_t)nx * ny * nz;
  bool dev_a = false;
  if ((rc = check_ptr(a, dev, 16, "a", &dev_a))) return rc;
  cudaStream_t s = g_stream;
  double2* d = reinterpret_cast<double2*>(a);
  if (!dev_a) {
    CK(cudaMallocAsync((void**)&d, sizeof(double2) * n, s));
    cudaError_t e = cudaMemcpyAsync(d, a, sizeof(double2) * n, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) {
      cudaFreeAsync(d, s);
      return cuda_fail(e, "fft3d");
    }
  }
  cudaError_t e = launch_fft3d(d, nx, ny, nz, isign, Tw{ctx->twf, ctx->twd}, s);
  if (e == cudaSuccess && !dev_a) e = cudaMemcpyAsync(a, d, sizeof(double2) * n, cudaMemcpyDeviceToHost, s);
  if (!dev_a) cudaFreeAsync(d, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return cuda_fail(e, "fft3d");
  return SS3D_OK;
}

// ---------------------------------------------------------------- host jump-ahead
// State of the Park-Miller stream right after the first draw of row (j, k) of
// realization r: 16807^(11 + r D + d prefix(j, k)) s0 mod (2^31 - 1), the value
// the realization kernels start that row from.  Host arithmetic only, so that
// a host can plan and check a split of realizations over processes or GPUs.
extern "C" int ss3d_row_state(const int np[3], int igauss, int iseed, int64_t r, int j, int k, uint32_t* state) {
  if (!np || !state) return fail(SS3D_EINVAL, "NULL argument");
  if (np[0] < 1 || np[1] < 1 || np[2] < 1) return fail(SS3D_EINVAL, "grid sizes must be positive");
  if (j < 0 || j >= np[1] || k < 0 || k >= np[2] || r < 0) return fail(SS3D_EINVAL, "row or realization out of range");
  Geo g{};
  g.npx = np[0];
  g.npy = np[1];
  g.npz = np[2];
  g.nx = g.npx;
  g.ny = g.npy;
  g.nz = g.npz;
  g.H = g.npx >= 2 ? g.npx / 2 + 1 : 1;
  g.HP = (g.H + 1) & ~1;
  g = geo_for_np(g, igauss);
  const uint64_t M1 = (uint64_t)(PM_M - 1);
  uint64_t t = ((uint64_t)r % M1) * (g.D % M1) % M1;
  t = (t + (uint64_t)g.d * row_prefix(g, j, k)) % M1;
  uint64_t e = (11ull + t) % M1;
  uint32_t base = PM_A, acc = 1;
  while (e) {
    if (e & 1) acc = pm_mulmod(acc, base);
    base = pm_mulmod(base, base);
    e >>= 1;
  }
  *state = pm_mulmod(acc, seed0(iseed));
  return SS3D_OK;
}

// ---------------------------------------------------------------- debug hooks
namespace ss3d {
cudaError_t launch_debug_states(const Geo& g, const uint32_t* rowstates, const uint32_t* apow, uint32_t* out,
                                cudaStream_t st);
}

extern "C" int ss3d_debug_states(const ss3d_spectrum* sp, int iseed, int64_t r, int igauss, uint32_t* states) {
  if (!sp || !states) return fail(SS3D_EINVAL, "NULL argument");
  if (r < 0) return fail(SS3D_EINVAL, "r must be >= 0");
  DevCtx* ctx;
  int rc;
  if ((rc = get_ctx(&ctx))) return rc;
  Geo g = geo_for(sp, igauss != 0);
  cudaStream_t s = g_stream;
  const size_t nhalf = (size_t)g.npz * g.npy * g.H;
  uint32_t *rs = nullptr, *apow = nullptr, *o = nullptr;
  CK(cudaMalloc(&rs, sizeof(uint32_t) * g.npy * g.npz));
  CK(cudaMalloc(&apow, sizeof(uint32_t) * g.npx));
  CK(cudaMalloc(&o, sizeof(uint32_t) * nhalf));
  cudaError_t e = launch_rowstates(g, seed0(iseed), r, 1, ctx->ptab, rs, apow, s);
  if (e == cudaSuccess) e = launch_debug_states(g, rs, apow, o, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(states, o, sizeof(uint32_t) * nhalf, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(rs);
  cudaFree(apow);
  cudaFree(o);
  if (e != cudaSuccess) return cuda_fail(e, "debug_states");
  return SS3D_OK;
}

extern "C" int ss3d_debug_coefficients(const ss3d_spectrum* sp, int iseed, int64_t r, int igauss, int precision,
                                       double* coef) {
  if (!sp || !coef) return fail(SS3D_EINVAL, "NULL argument");
  if (r < 0) return fail(SS3D_EINVAL, "r must be >= 0");
  DevCtx* ctx;
  int rc;
  if ((rc = get_ctx(&ctx))) return rc;
  const bool dbl = precision == SS3D_FP64;
  Geo g = geo_for(sp, igauss != 0);
  cudaStream_t s = g_stream;
  const size_t nh = (size_t)g.npz * g.npy * g.HP;
  uint32_t *rs = nullptr, *apow = nullptr;
  void* w = nullptr;
  CK(cudaMalloc(&rs, sizeof(uint32_t) * g.npy * g.npz));
  CK(cudaMalloc(&apow, sizeof(uint32_t) * g.npx));
  CK(cudaMalloc(&w, (dbl ? sizeof(double2) : sizeof(float2)) * nh));
  cudaError_t e = launch_rowstates(g, seed0(iseed), r, 1, ctx->ptab, rs, apow, s);
  if (e == cudaSuccess) {
    if (dbl)
      e = launch_gen<double>(g, sp->amp64, rs, apow, (double2*)w, 0, 1, s);
    else
      e = launch_gen<float>(g, sp->amp32, rs, apow, (float2*)w, 0, 1, s);
  }
  std::vector<char> h((dbl ? sizeof(double2) : sizeof(float2)) * nh);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), w, h.size(), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  cudaFree(rs);
  cudaFree(apow);
  cudaFree(w);
  if (e != cudaSuccess) return cuda_fail(e, "debug_coefficients");
  for (size_t row = 0; row < (size_t)g.npz * g.npy; row++)
    for (int i = 0; i < g.H; i++) {
      size_t src = row * g.HP + i, dst = row * g.H + i;
      if (dbl) {
        const double2* p = (const double2*)h.data();
        coef[2 * dst] = p[src].x;
        coef[2 * dst + 1] = p[src].y;
      } else {
        const float2* p = (const float2*)h.data();
        coef[2 * dst] = p[src].x;
        coef[2 * dst + 1] = p[src].y;
      }
    }
  return SS3D_OK;
}

// ---------------------------------------------------------------- helpers of the allocation-free entry point
int ss3d::set_error(int code, const char* msg) { return fail(code, "%s", msg); }
cudaStream_t ss3d::current_stream() { return g_stream; }
int ss3d::spectrum_view(const ss3d_spectrum* sp, NoallocView* v) {
  if (!sp || !sp->amp32 || !sp->amp64) return 1;
  v->dev = sp->dev;
  v->geo = sp->geo;
  v->amp64 = sp->amp64;
  v->amp32 = sp->amp32;
  return 0;
}

// helpers of the batched form (ss3d_batch.cu)
int ss3d::batch_ctx(int dev, Tw* tw, const uint32_t** ptab) {
  (void)dev;
  DevCtx* ctx;
  if (int rc = get_ctx(&ctx)) return rc;
  *tw = Tw{ctx->twf, ctx->twd};
  *ptab = ctx->ptab;
  return SS3D_OK;
}
int ss3d::batch_geo(const ss3d_spectrum* sp, int igauss, Geo* g, const float** amp32) {
  int dev = -1;
  if (!sp || !sp->amp32 || cudaGetDevice(&dev) != cudaSuccess || dev != sp->dev) return 1;
  *g = geo_for(sp, igauss);
  *amp32 = sp->amp32;
  return 0;
}

// model helpers shared with the conditioning module
void ss3d::setrot_public(const ss3d_struct& s, double rot[3][3], double axes[3][3]) { setrot_rc(s, rot, axes); }
void ss3d::model_public(const ss3d_struct* st, int nst, double nugget, Model& m) { build_model(st, nst, nugget, m); }

// ---------------------------------------------------------------- autotuner
namespace ss3d {
extern int g_variant[3][2][16];
}

extern "C" int ss3d_autotune(const ss3d_spectrum* sp, int igauss, int precision, int nreal, int chosen[3]) {
  if (!sp) return fail(SS3D_EINVAL, "spectrum is NULL");
  if (precision != SS3D_FP64 && precision != SS3D_FP32) return fail(SS3D_EINVAL, "unknown precision");
  if (nreal < 1) return fail(SS3D_EINVAL, "nreal must be >= 1");
  const Geo& g = sp->geo;
  const int p = precision == SS3D_FP32 ? 1 : 0;
  // the transform length each kernel kind runs at for this grid
  int L[3] = {-1, -1, -1};
  if (g.npz > 1) {
    L[1] = ilog2i(g.npz);
    if (g.npy > 1) L[0] = ilog2i(g.npy);
  } else if (g.npy > 1) {
    L[1] = ilog2i(g.npy);
  }
  if (g.npx > 1) L[2] = ilog2i(g.npx) - 1;
  // the middle pass and the synthesis pass may share a length: tune them jointly then
  const size_t M = (size_t)g.nx * g.ny * g.nz;
  float* out = nullptr;
  CK(cudaMalloc(&out, sizeof(float) * M * nreal));
  const bool prof_was = g_prof;
  double best[3] = {1e30, 1e30, 1e30};
  double fused_ms = 1e30;   // row variant 5: middle and row passes in one kernel
  int bestv[3] = {0, 0, 0};
  int rc = SS3D_OK;
  // variants per kind: 0-3 everywhere, FP32 column passes also 4-7 (two
  // lines per thread), the FP32 middle pass also 8-9 (tiles staged by bulk
  // tensor copies), the row pass also 4 (rows held in warps) and, in FP32, 5
  // (middle and row passes fused over a cluster) and 6 (two rows per lane on
  // packed FP32); a kind with fewer variants runs its variant v mod 4 meanwhile
  const int nvk[3] = {precision == SS3D_FP32 ? 10 : 4, precision == SS3D_FP32 ? 8 : 4,
                      precision == SS3D_FP32 ? 7 : 5};
  const int nv = std::max(nvk[0], nvk[2]);
  auto vk = [&](int k, int v) { return v < nvk[k] ? v : v % 4; };
  for (int v = 0; v < nv && rc == SS3D_OK; v++) {
    for (int k = 0; k < 3; k++)
      if (L[k] >= 0) g_variant[k][p][L[k]] = vk(k, v);
    rc = ss3d_realize(sp, 1, 0, nreal, igauss, precision, out, SS3D_OUT_F32, nullptr);   // warm up
    if (rc) break;
    g_prof = true;
    for (int q = 0; q < SS3D_NSTAGE; q++) g_prof_ms[q] = 0;
    for (int rep = 0; rep < 2 && rc == SS3D_OK; rep++)
      rc = ss3d_realize(sp, 1, 0, nreal, igauss, precision, out, SS3D_OUT_F32, nullptr);
    g_prof = prof_was;
    if (rc) break;
    const double ms[3] = {g_prof_ms[2], g_prof_ms[1], g_prof_ms[3]};   // stage 2 middle, 1 synthesis, 3 rows
    // row variant 5 runs the middle pass inside the row stage: it competes
    // with the best middle + row pair below, not with either pass alone
    const bool joint = L[2] >= 0 && vk(2, v) == 5;
    if (joint && L[0] >= 0 && g_prof_ms[2] == 0.0) {
      fused_ms = std::min(fused_ms, ms[2]);
      if (L[1] >= 0 && ms[1] < best[1]) {
        best[1] = ms[1];
        bestv[1] = vk(1, v);
      }
      continue;
    }
    for (int k = 0; k < 3; k++)
      if (L[k] >= 0 && ms[k] < best[k] && !(k == 2 && vk(2, v) == 5)) {
        best[k] = ms[k];
        bestv[k] = vk(k, v);
      }
  }
  if (fused_ms < best[0] + best[2]) bestv[2] = 5;
  for (int k = 0; k < 3; k++)
    if (L[k] >= 0) g_variant[k][p][L[k]] = bestv[k];
  for (int q = 0; q < SS3D_NSTAGE; q++) g_prof_ms[q] = 0;
  cudaFree(out);
  if (chosen)
    for (int k = 0; k < 3; k++) chosen[k] = bestv[k];
  return rc;
}

extern "C" int ss3d_set_variant(int kind, int precision, int logn, int variant) {
  // 4-7: FP32 two-line column tiles; 8, 9: FP32 middle pass staged by bulk
  // tensor copies (one and two lines per thread); 4 of the row pass: rows held
  // in warps; 5 of the FP32 row pass: middle and row passes fused over a
  // cluster; 6 of the FP32 row pass: two rows per lane on packed FP32
  const int vmax = kind == 2 ? (precision == SS3D_FP32 ? 6 : 4) : (precision == SS3D_FP32 ? (kind == 0 ? 9 : 7) : 3);
  if (kind < 0 || kind > 2 || (precision != SS3D_FP64 && precision != SS3D_FP32) || logn < 0 || logn > 15 ||
      variant < 0 || variant > vmax)
    return fail(SS3D_EINVAL, "invalid variant selection");
  g_variant[kind][precision == SS3D_FP32 ? 1 : 0][logn] = variant;
  return SS3D_OK;
}
