// ss3d_noalloc.cu -- realization entry point that allocates no device memory.
//
// Some callers cannot call cudaMalloc at the point where they want
// realizations: a host application that has already handed the GPU's memory
// to its own pool (a serving process that reserves HBM up front for its
// request queue) gets an allocation failure or fragments that pool, and a
// latency-sensitive loop cannot afford cudaMalloc/cudaFree, which synchronise
// the device and stall every stream in flight.  ss3d_realize_noalloc runs the
// same kernels as ss3d_realize, but all of its scratch memory (the complex
// half-spectrum work grid, the Park-Miller row states and offsets, the
// twiddle and jump-ahead tables) lives in one file-scope __device__ array of
// fixed size, reserved on every GPU that loads this library until the process
// exits.
//
// Limits and rules:
//  * the scratch array is SS3D_NOALLOC_SCRATCH_BYTES (64 MiB); one call needs
//    about nz * npy * (npx/2 + 2) * 8 bytes (FP32, 16 for FP64) plus 0.5 MB of
//    tables.  A 128^3 grid on its 256^3 periodic grid fits in FP32 (34 MB) but
//    not in FP64 (68 MB), and the 256^3 grid on 512^3 fits in neither; a grid
//    that does not fit is rejected with SS3D_ETOOLARGE and a message giving
//    the bytes it would need;
//  * out must be device memory of the device that holds the spectrum, which
//    must also be the current device (host pointers and other devices are
//    rejected with SS3D_EINVAL before any work is issued);
//  * the first call on a device fills the twiddle and jump-ahead tables of the
//    array for that device (a host-to-device copy followed by a device
//    synchronisation); make that first call before any stream capture begins;
//  * every call shares the one array and overwrites it: calls that overlap on
//    the GPU (two host threads, or two streams) race and corrupt each other.
//    Nothing in the array needs to start at zero: every element a kernel reads
//    was written earlier in the same call.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/specsim3d_gpu.h"
#include "ss3d_internal.h"

using namespace ss3d;

namespace {

constexpr size_t kScratchBytes = (size_t)SS3D_NOALLOC_SCRATCH_BYTES;
constexpr int kTwCount = (1 << (TW_LOG_MAX + 1)) - 1;   // twiddle entries, n = 1 .. 2^13
// every region starts on a 256-byte boundary (the kernels load 16-byte double2)
constexpr size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffTwF = 0;
constexpr size_t kOffTwD = up256(kOffTwF + sizeof(float2) * kTwCount);
constexpr size_t kOffPtab = up256(kOffTwD + sizeof(double2) * kTwCount);
constexpr size_t kOffFree = up256(kOffPtab + sizeof(uint32_t) * 3 * 2048);
static_assert(kOffTwD % 16 == 0 && kOffPtab % 16 == 0 && kOffFree % 256 == 0, "scratch regions must be aligned");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct DevScratch {
  bool ready = false;
  unsigned char* base = nullptr;
};
std::mutex g_mu;
DevScratch g_dev[64];

int fail(int code, const std::string& m) { return set_error(code, m.c_str()); }

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// once per device, with that device current: the device address of the array
// (the host-side name is only a stand-in) and the constant tables
int setup(int dev, unsigned char** base) {
  std::lock_guard<std::mutex> lk(g_mu);
  DevScratch& d = g_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return fail(SS3D_ECUDA, std::string("cudaGetSymbolAddress of the scratch array: ") + cudaGetErrorString(e));
    std::vector<float2> hf(kTwCount);
    std::vector<double2> hd(kTwCount);
    for (int L = 0; L <= TW_LOG_MAX; ++L) {
      int n = 1 << L;
      for (int m = 0; m < n; ++m) {
        long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)m / (long double)n;
        hd[n - 1 + m] = make_double2((double)cosl(ang), (double)sinl(ang));
        hf[n - 1 + m] = make_float2((float)cosl(ang), (float)sinl(ang));
      }
    }
    std::vector<uint32_t> ht(3 * 2048);
    uint32_t b = PM_A;
    for (int l = 0; l < 3; ++l) {
      uint32_t acc = 1;
      for (int v = 0; v < 2048; ++v) {
        ht[l * 2048 + v] = acc;
        acc = pm_mulmod(acc, b);
      }
      b = acc;
    }
    unsigned char* s = (unsigned char*)p;
    e = cudaMemcpy(s + kOffTwF, hf.data(), sizeof(float2) * kTwCount, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s + kOffTwD, hd.data(), sizeof(double2) * kTwCount, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s + kOffPtab, ht.data(), sizeof(uint32_t) * 3 * 2048, cudaMemcpyHostToDevice);
    // a copy from pageable memory may return before its DMA ends, and the
    // kernels run on the caller's stream, which need not order behind the
    // legacy stream: wait for the copies before the first launch
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return fail(SS3D_ECUDA, std::string("scratch table set-up: ") + cudaGetErrorString(e));
    d.base = s;
    d.ready = true;
  }
  *base = d.base;
  return SS3D_OK;
}

}  // namespace

extern "C" int ss3d_realize_noalloc(const ss3d_spectrum* sp, int iseed, int64_t r_first, int nreal, int igauss,
                                    int precision, void* out, int out_dtype) {
  NoallocView v;
  if (!sp) return fail(SS3D_EINVAL, "spectrum is NULL");
  if (spectrum_view(sp, &v)) return fail(SS3D_EINVAL, "invalid spectrum handle");
  if (nreal < 0 || r_first < 0) return fail(SS3D_EINVAL, "nreal and r_first must be >= 0");
  if (igauss != 0 && igauss != 1) return fail(SS3D_EINVAL, "igauss must be 0 or 1");
  if (precision != SS3D_FP64 && precision != SS3D_FP32) return fail(SS3D_EINVAL, "unknown precision");
  if (out_dtype != SS3D_OUT_F32 && out_dtype != SS3D_OUT_F64) return fail(SS3D_EINVAL, "unknown out_dtype");
  if (nreal == 0) return SS3D_OK;
  if (!out) return fail(SS3D_EINVAL, "out is NULL");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) return fail(SS3D_ECUDA, "no current CUDA device");
  if (dev != v.dev) {
    char buf[160];
    snprintf(buf, sizeof buf, "the spectrum lives on device %d but device %d is current", v.dev, dev);
    return fail(SS3D_EINVAL, buf);
  }
  Geo g = v.geo;
  const size_t oel = out_dtype == SS3D_OUT_F32 ? 4 : 8;
  bool dev_out = false;
  if (int rc = check_ptr(out, dev, (g.nx % 2 == 0 ? 2 : 1) * oel, "out", &dev_out)) return rc;
  if (!dev_out) return fail(SS3D_EINVAL, "ss3d_realize_noalloc needs a device output pointer");
  const bool dbl = precision == SS3D_FP64;
  const int maxl = dbl ? MAX_LOGN_D : MAX_LOGN_F;
  auto lg = [](int n) { int l = 0; while ((1 << l) < n) ++l; return l; };
  if ((g.npx > 1 && lg(g.npx) - 1 > maxl) || lg(g.npy) > maxl || lg(g.npz) > maxl)
    return fail(SS3D_ETOOLARGE, "periodic axis longer than the supported transform length");
  g.d = igauss ? 2 : 1;
  const uint64_t N = (uint64_t)g.npx * g.npy * g.npz;
  const uint64_t nself = (uint64_t)(g.npx >= 2 ? 2 : 1) * (g.npy >= 2 ? 2 : 1) * (g.npz >= 2 ? 2 : 1);
  g.D = (uint64_t)g.d * ((N + nself) / 2);
  // one realization at a time; the work grid holds the planes that survive the
  // first (pruned) pass: nz planes when there is a z pass, else the whole plane
  const size_t planes = g.npz > 1 ? (size_t)g.nz : 1;
  const size_t cel = dbl ? sizeof(double2) : sizeof(float2);
  const size_t need_work = planes * g.npy * g.HP * cel;
  const size_t off_rs = kOffFree;
  const size_t off_apow = al256(off_rs + sizeof(uint32_t) * g.npy * g.npz);
  const size_t off_work = al256(off_apow + sizeof(uint32_t) * g.npx);
  const size_t need = off_work + need_work;
  if (need > kScratchBytes) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "grid needs %zu bytes of scratch; ss3d_realize_noalloc has %zu (use ss3d_realize for larger grids)", need,
             kScratchBytes);
    return fail(SS3D_ETOOLARGE, buf);
  }
  unsigned char* base = nullptr;
  int rc = setup(dev, &base);
  if (rc) return rc;
  Tw tw{(const float2*)(base + kOffTwF), (const double2*)(base + kOffTwD)};
  const uint32_t* ptab = (const uint32_t*)(base + kOffPtab);
  uint32_t* rs = (uint32_t*)(base + off_rs);
  uint32_t* apow = (uint32_t*)(base + off_apow);
  void* work = base + off_work;
  int64_t a = iseed < 0 ? -(int64_t)iseed : (int64_t)iseed;
  const uint32_t s0 = (uint32_t)(a % 2147483646LL + 1);
  const size_t M = (size_t)g.nx * g.ny * g.nz;
  cudaStream_t st = current_stream();
  const unsigned long long pipes0 = g_pipe_launches.load();
  for (int r = 0; r < nreal && e == cudaSuccess; ++r) {
    e = launch_rowstates(g, s0, r_first + r, 1, ptab, rs, r == 0 ? apow : nullptr, st);
    void* dst = (char*)out + (size_t)r * M * oel;
    if (e == cudaSuccess) {
      if (dbl)
        e = launch_realize<double>(g, v.amp64, rs, apow, (double2*)work, 0, 1, dst, out_dtype, nullptr, nullptr, tw,
                                   true, st);
      else
        e = launch_realize<float>(g, v.amp32, rs, apow, (float2*)work, 0, 1, dst, out_dtype, nullptr, nullptr, tw,
                                  true, st);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(SS3D_ECUDA, std::string("realize_noalloc: ") + cudaGetErrorString(e));
  }
  if (g_pipe_launches.load() != pipes0 && pipe_error_take(st))
    return fail(SS3D_ECUDA, "realize_noalloc: a bulk-copy wait of the middle pass timed out");
  return SS3D_OK;
}
