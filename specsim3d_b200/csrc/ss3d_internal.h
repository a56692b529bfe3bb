// ss3d_internal.h -- host/device shared declarations of the CUDA library
// (not part of the public C ABI in include/specsim3d_gpu.h).
#pragma once
#include <atomic>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>

#include "ss3d_device.cuh"
#include "../../include/specsim3d_gpu.h"

namespace ss3d {

constexpr int MAXST = 10;          // f90:93
constexpr int MAX_LOGN_F = 12;     // longest axis kept in shared memory, float
constexpr int MAX_LOGN_D = 11;     // longest axis kept in shared memory, double
constexpr int TW_LOG_MAX = 13;     // twiddle tables for n = 1 .. 2^13

// Twiddle tables: for n = 2^L the table e^{-2 pi i m / n}, m in [0, n), starts
// at offset n - 1.
struct Tw {
  const float2* f;
  const double2* d;
};

// Variogram model after setrot (f90:95-139), in kernel-parameter form.
struct Model {
  int nst;
  double nugget;
  int itype[MAXST];
  double sill[MAXST], ahmax[MAXST];
  double rot[MAXST][9];   // row-major rot(r, c) -> rot[s][3*r + c]
};

// covariance, f90:153-178
__host__ __device__ inline double covariance(const Model& m, double dx, double dy, double dz) {
  double c = 0.0;
  if (dx == 0.0 && dy == 0.0 && dz == 0.0) c = m.nugget;
  for (int i = 0; i < m.nst; i++) {
    const double* r = m.rot[i];
    double rx = r[0] * dx + r[1] * dy + r[2] * dz;
    double ry = r[3] * dx + r[4] * dy + r[5] * dz;
    double rz = r[6] * dx + r[7] * dy + r[8] * dz;
    double h = sqrt(rx * rx + ry * ry + rz * rz);
    double hr = h / m.ahmax[i];
    if (m.itype[i] == 1) {
      if (hr < 1.0) c = c + m.sill[i] * (1.0 - 1.5 * hr + 0.5 * (hr * hr * hr));
    } else if (m.itype[i] == 2) {
      c = c + m.sill[i] * exp(-3.0 * hr);
    } else {
      c = c + m.sill[i] * exp(-(3.0 * hr * hr));
    }
  }
  return c;
}

// Spectrum diagnostics, f90:1275-1292, accumulated over the full spectrum
struct SpecPartial {
  double maximag, maxreal, spos, sneg;
};

// Stage markers of one realize call (CUDA events recorded between stages)
struct Marks {
  bool on = false;
  int n = 0;
  int stage[16];
  cudaEvent_t ev[16];
};
void mark(Marks* m, int stage, cudaStream_t st);   // records an event opening `stage`
// Raises a kernel's dynamic shared memory limit on the current device once per
// size: changing a function attribute while instances of it run on other
// streams can make the call wait for them, so repeated calls return at once.
cudaError_t func_smem(const void* kernel, size_t bytes);
// one kernel of each translation unit with kernels: its module holds them all
const void* module_anchor_fft();
const void* module_anchor_cond();
const void* module_anchor_vario();
const void* module_anchor_batch();
extern std::atomic<unsigned long long> g_launch_count;   // kernels launched by the library (all threads)
// launches of kernels that stage tiles with bulk copies and bounded waits;
// after work that contains one, pipe_error_take reads (and clears) the flag a
// timed-out wait leaves, synchronising the stream
extern std::atomic<unsigned long long> g_pipe_launches;
bool pipe_error_take(cudaStream_t st);

// ---- launchers (ss3d_fft.cu); all return cudaError_t of the last launch
cudaError_t launch_spectrum(const Model& m, const double d[3], const Geo& g, double2* work, double* amp64,
                            float* amp32, SpecPartial* part, int npart_max, SpecPartial* result, Tw tw,
                            cudaStream_t st);
int spectrum_parts(const Geo& g);   // partial-sum entries of a spectrum build (npart_max + 1)
cudaError_t launch_rowstates(const Geo& g, uint32_t s0, long long r_first, int nreal, const uint32_t* ptab,
                             uint32_t* rowstates, uint32_t* apow, cudaStream_t st);
// out_kind: 0 float output, 1 double output; first_done (may be NULL) is
// recorded on st once the first pass (synthesis) has been enqueued
template <typename R>
cudaError_t launch_realize(const Geo& g, const R* amp, const uint32_t* rowstates, const uint32_t* apow,
                           cpx_t<R>* work, long long wstride, int nreal, void* out, int out_kind,
                           double* part, int* nblk_per_r, Tw tw, bool fused, cudaStream_t st,
                           Marks* marks = nullptr, cudaEvent_t first_done = nullptr);
template <typename R>
cudaError_t launch_gen(const Geo& g, const R* amp, const uint32_t* rowstates, const uint32_t* apow,
                       cpx_t<R>* work, long long wstride, int nreal, cudaStream_t st);
cudaError_t launch_fft3d(double2* a, int nx, int ny, int nz, int isign, Tw tw, cudaStream_t st);
cudaError_t launch_reduce_zstats(const double* part, int nblk_per_r, int nreal, double* zsum, cudaStream_t st);
int realize_part_blocks(const Geo& g, bool dbl);

// ---- helpers of the allocation-free entry point (ss3d_api.cu)
struct NoallocView {
  int dev;              // device that holds the amplitudes
  Geo geo;
  const double* amp64;
  const float* amp32;
};
int set_error(int code, const char* msg);     // sets the message returned by ss3d_last_error
// Where caller memory p lives.  *is_dev becomes true for device (or managed)
// memory, false for host memory (pageable or pinned), which the library only
// reaches through copies.  Device memory must belong to device `dev` and start
// on a multiple of `align` bytes (the kernels store 2-element vectors into
// output rows of even length); otherwise SS3D_EINVAL with a message naming
// `what`, before any work is issued.
int check_ptr(const void* p, int dev, size_t align, const char* what, bool* is_dev);
void setrot_public(const ss3d_struct& s, double rot[3][3], double axes[3][3]);
void model_public(const ss3d_struct* st, int nst, double nugget, Model& m);
cudaStream_t current_stream();                // stream selected with ss3d_set_stream

}  // namespace ss3d

struct ss3d_spectrum;
namespace ss3d {
int spectrum_view(const ss3d_spectrum* sp, NoallocView* v);
int64_t realize_bytes_for(const int np[3], const int n[3], int nreal, int precision, int host_out);
int batch_ctx(int dev, Tw* tw, const uint32_t** ptab);   // twiddle and jump tables of the current device
// Maps up to `bytes` of device memory into the stream-ordered pool of the
// current device (one allocation, freed at once; the pool keeps it mapped), so
// that later allocations up to that total find mapped pages; best effort:
// halves the request on failure.  Returns the bytes mapped.
size_t pool_premap(size_t bytes);
// geometry of a spectrum for igauss and its FP32 amplitudes; 1 if the handle is
// invalid or lives on another device than the current one
int batch_geo(const ss3d_spectrum* sp, int igauss, Geo* g, const float** amp32);
}  // namespace ss3d
