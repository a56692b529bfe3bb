// ss3d_vario.cu -- experimental semivariograms over all node pairs
// (reference: npair_count f90:394-402, vario_lag f90:405-431, task loop of
// vario_report f90:462-480).
//
// gamma(l) = 0.5 * sum over all node pairs (p, p + l s) of (f(p + l s) - f(p))^2
//            / npair(l),   npair = prod_a (n_a - |l s_a|)  (0 if any |l s_a| >= n_a)
//
// The pair count is exact integer arithmetic on the host.  The sums are FP64.
// Since gamma(l s) = gamma(-l s) (the same pairs read in the other order), a
// direction is normalised so that its leading march component is positive.
//
// Kernel layout: a CTA owns a sheared slab of base points
//     p(t, m) = q0 + t u + m v,   t in [0, 32) lanes,  m in [m0, m0 + T)
// and stages f on p(t, m) for m in [m0, m0 + T + L mu) in shared memory
// (s[m][t], coalesced loads along x).  The partner of base (t, m) at lag l is
// (t, m + l mu).  Two cases:
//   * general (s has a y or z component): u = e_x, v = s, mu = 1; the slab is
//     keyed by the residue r of the leading axis and the virtual start q
//     (points outside the grid are masked);
//   * pure x (s = (sx, 0, 0)): u = e_y, v = e_x, mu = sx.
// Each line t meets the grid on one interval of m, so a pair is valid iff its
// base is valid and m + l mu lies before the end of that interval.  Warp w of
// the CTA accumulates the lags l = l0 + w, l0 + w + NW, ... in registers; the
// per-CTA lag sums go to a partial buffer reduced in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/specsim3d_gpu.h"
#include "ss3d_internal.h"

namespace ss3d {

constexpr int VT = 128;      // base march steps per CTA
constexpr int VNW = 8;       // warps per CTA
constexpr int VLPT = 16;     // lags per thread per launch
constexpr int VLCH = VNW * VLPT;  // lags per launch (128)
constexpr int VPW = 128;     // lags * mu per launch at most: partner window VT + VPW - 1 steps
constexpr int VP = 33;       // shared-memory pitch (lanes + 1)

struct VarioGeo {
  int nx, ny, nz;
  int mode;          // 0 general (v = s), 1 pure x (v = e_x, mu = sx)
  int sx, sy, sz;    // normalised direction
  int mu;            // partner offset per lag along the march
  int a;             // general: leading axis 1 = y, 2 = z
  int sig;           // general: s_a > 0
  int qx_lo, nqx;    // general: virtual start range along x (32 per tile); pure x: row tiles
  int qb_lo, nqb;    // general: virtual start range along the other axis
  int mmax;          // march length bound
  int nmb;           // march blocks of VT
  int ncta;          // CTAs per realization
};

__host__ __device__ __forceinline__ long long floordiv(long long a, long long b) {  // b > 0
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}
__host__ __device__ __forceinline__ long long ceildiv(long long a, long long b) { return -floordiv(-a, b); }

// Line of lane t of CTA cta: start point (linear index base), step per march
// index (linear), the valid march interval [vlo, vhi) where the point is
// inside the grid, and the first base march index m0 of the CTA.
__device__ __forceinline__ void lane_line(const VarioGeo& G, int cta, int t, int& vlo, int& vhi, long long& base,
                                          long long& step, int& m0) {
  int mb = cta % G.nmb;
  int rest = cta / G.nmb;
  m0 = mb * VT;
  long long x0, y0, z0, dx, dy, dz;
  if (G.mode == 1) {
    int jt = rest % G.nqx;
    int k = rest / G.nqx;
    x0 = 0;
    y0 = (long long)jt * 32 + t;
    z0 = k;
    dx = 1;
    dy = 0;
    dz = 0;
  } else {
    int xt = rest % G.nqx;
    rest /= G.nqx;
    int qb = G.qb_lo + rest % G.nqb;
    int r = rest / G.nqb;
    x0 = (long long)G.qx_lo + (long long)xt * 32 + t;
    if (G.a == 2) {
      z0 = r;
      y0 = qb;
    } else {
      y0 = r;
      z0 = qb;
    }
    dx = G.sx;
    dy = G.sy;
    dz = G.sz;
  }
  long long lo = 0, hi = G.mmax;
  auto clip = [&](long long c0, long long dc, long long n) {
    if (dc == 0) {
      if (c0 < 0 || c0 >= n) hi = lo;
    } else if (dc > 0) {
      lo = max(lo, ceildiv(-c0, dc));
      hi = min(hi, floordiv(n - 1 - c0, dc) + 1);
    } else {
      const long long e = -dc;
      lo = max(lo, ceildiv(c0 - n + 1, e));
      hi = min(hi, floordiv(c0, e) + 1);
    }
  };
  clip(x0, dx, G.nx);
  clip(y0, dy, G.ny);
  clip(z0, dz, G.nz);
  if (hi < lo) hi = lo;
  vlo = (int)lo;
  vhi = (int)hi;
  base = x0 + (long long)G.nx * (y0 + (long long)G.ny * z0);
  step = dx + (long long)G.nx * (dy + (long long)G.ny * dz);
}

// Shared memory: base window sb[VT][VP] (march m0 .. m0+VT-1) and partner
// window sp[VT+VPW-1][VP] (march ps .. , ps = m0 + l0 mu).  For base m and lag
// l in [l0, l0+nl), the partner index m + l mu - ps lies in
// [0, VT - 1 + (nl - 1) mu] and nl * mu <= VPW, so every read is inside sp.
__global__ void __launch_bounds__(32 * VNW) k_vario(VarioGeo G, const double* __restrict__ f, long long fstride,
                                                    int l0, int nl, double* __restrict__ part) {
  extern __shared__ __align__(16) double smv[];
  double* sb = smv;
  double* spw = smv + VT * VP;
  const int r = blockIdx.y;
  const int cta = blockIdx.x;
  const int t = threadIdx.x & 31, w = threadIdx.x >> 5;
  const double* fr = f + (long long)r * fstride;
  const int pspan = VT + (nl - 1) * G.mu;
  int vlo, vhi, m0;
  long long base, step;
  lane_line(G, cta, t, vlo, vhi, base, step, m0);
  const int ps = m0 + l0 * G.mu;
  if (G.mode == 0) {
    // lanes t are consecutive x: coalesced along each march step
    for (int q = w; q < VT; q += VNW) {
      const int m = m0 + q;
      sb[q * VP + t] = (m >= vlo && m < vhi) ? __ldg(fr + base + (long long)m * step) : 0.0;
    }
    for (int q = w; q < pspan; q += VNW) {
      const int m = ps + q;
      spw[q * VP + t] = (m >= vlo && m < vhi) ? __ldg(fr + base + (long long)m * step) : 0.0;
    }
  } else {
    // pure x: line t is row t of the tile; lanes run along x for coalescing
    for (int row = w; row < 32; row += VNW) {
      int rvlo, rvhi, rm0;
      long long rbase, rstep;
      lane_line(G, cta, row, rvlo, rvhi, rbase, rstep, rm0);
      for (int q = t; q < VT; q += 32) {
        const int m = m0 + q;
        sb[q * VP + row] = (m >= rvlo && m < rvhi) ? __ldg(fr + rbase + m) : 0.0;
      }
      for (int q = t; q < pspan; q += 32) {
        const int m = ps + q;
        spw[q * VP + row] = (m >= rvlo && m < rvhi) ? __ldg(fr + rbase + m) : 0.0;
      }
    }
  }
  __syncthreads();
  double acc[VLPT];
#pragma unroll
  for (int q = 0; q < VLPT; ++q) acc[q] = 0.0;
  const int mb0 = max(m0, vlo), mb1 = min(m0 + VT, vhi);
  for (int m = mb0; m < mb1; ++m) {
    const double b = sb[(m - m0) * VP + t];
#pragma unroll
    for (int q = 0; q < VLPT; ++q) {
      const int li = w + q * VNW;
      const int mp = m + (l0 + li) * G.mu;
      if (li < nl && mp < vhi) {
        const double d = spw[(mp - ps) * VP + t] - b;
        acc[q] = fma(d, d, acc[q]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < VLPT; ++q) {
    double v = acc[q];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    const int li = w + q * VNW;
    if (t == 0 && li < nl) part[((long long)r * G.ncta + cta) * VLCH + li] = v;
  }
}

// gam[(l-1) + nlagmax*(d + ndir*r)] = 0.5 * sum_cta part / npairs, fixed order
__global__ void k_vario_reduce(const double* __restrict__ part, int ncta, int l0, int nl, int d, int ndir,
                               int nlagmax, const long long* __restrict__ npairs, double* gam, int rbase) {
  const int r = blockIdx.y;
  const int li = blockIdx.x;
  __shared__ double red[256];
  double s = 0.0;
  for (int c = threadIdx.x; c < ncta; c += 256) s += part[((long long)r * ncta + c) * VLCH + li];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if (threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const int l = l0 + li;
    const long long np = npairs[li];
    gam[(l - 1) + (long long)nlagmax * (d + (long long)ndir * (rbase + r))] = np > 0 ? 0.5 * red[0] / (double)np : 0.0;
  }
}

}  // namespace ss3d

using namespace ss3d;

namespace {
long long npair_count(int nx, int ny, int nz, long long lx, long long ly, long long lz) {
  if (llabs(lx) >= nx || llabs(ly) >= ny || llabs(lz) >= nz) return 0;
  return (long long)(nx - llabs(lx)) * (ny - llabs(ly)) * (nz - llabs(lz));
}
}  // namespace

extern "C" int ss3d_vario(const double* res, const int n[3], int nreal, int ndir, const int* sx, const int* sy,
                          const int* sz, const int* nlag, double* gam, int64_t* npairs) {
  if (!res || !n || !sx || !sy || !sz || !nlag || !gam) return set_error(SS3D_EINVAL, "NULL argument");
  if (n[0] < 1 || n[1] < 1 || n[2] < 1 || nreal < 0 || ndir < 0) return set_error(SS3D_EINVAL, "invalid sizes");
  int nlagmax = 0;
  for (int d = 0; d < ndir; d++) {
    if (nlag[d] < 0) return set_error(SS3D_EINVAL, "nlag must be >= 0");
    nlagmax = std::max(nlagmax, nlag[d]);
  }
  const int nx = n[0], ny = n[1], nz = n[2];
  // host pair counts (exact), the reference's npair_count
  std::vector<long long> np_all((size_t)std::max(1, nlagmax) * std::max(1, ndir), 0);
  for (int d = 0; d < ndir; d++)
    for (int l = 1; l <= nlag[d]; l++)
      np_all[(l - 1) + (size_t)nlagmax * d] = npair_count(nx, ny, nz, (long long)l * sx[d], (long long)l * sy[d],
                                                          (long long)l * sz[d]);
  if (npairs)
    for (size_t q = 0; q < np_all.size() && q < (size_t)nlagmax * ndir; q++) npairs[q] = np_all[q];
  const size_t M = (size_t)nx * ny * nz;
  const size_t ngam = (size_t)nlagmax * ndir * nreal;
  if (ngam == 0) return SS3D_OK;
  cudaStream_t st = current_stream();
  int cur_dev = 0;
  if (cudaGetDevice(&cur_dev) != cudaSuccess) return set_error(SS3D_ECUDA, "no current CUDA device");
  bool dev_in = false, dev_gam = false;
  if (int rc = check_ptr(res, cur_dev, sizeof(double), "res", &dev_in)) return rc;
  if (int rc = check_ptr(gam, cur_dev, sizeof(double), "gam", &dev_gam)) return rc;
  const double* fdev = res;
  double* fbuf = nullptr;
  double* gdev = nullptr;
  double* part = nullptr;
  long long* npdev = nullptr;
  cudaError_t e = cudaSuccess;
  if (!dev_in) {
    e = cudaMalloc(&fbuf, sizeof(double) * M * nreal);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fbuf, res, sizeof(double) * M * nreal, cudaMemcpyHostToDevice, st);
    fdev = fbuf;
  }
  if (e == cudaSuccess) e = cudaMalloc(&gdev, sizeof(double) * ngam);
  if (e == cudaSuccess) e = cudaMemsetAsync(gdev, 0, sizeof(double) * ngam, st);
  if (e == cudaSuccess) e = cudaMalloc(&npdev, sizeof(long long) * VLCH);
  // largest partial buffer over directions
  size_t part_elems = 0;
  std::vector<VarioGeo> geos(ndir);
  for (int d = 0; d < ndir && e == cudaSuccess; d++) {
    VarioGeo G{};
    G.nx = nx;
    G.ny = ny;
    G.nz = nz;
    int a = sx[d], b = sy[d], c = sz[d];
    // normalise the sign: leading non-zero of (z, y, x) positive
    int lead = c != 0 ? c : (b != 0 ? b : a);
    if (lead < 0) {
      a = -a;
      b = -b;
      c = -c;
    }
    G.sx = a;
    G.sy = b;
    G.sz = c;
    if (a == 0 && b == 0 && c == 0) {
      G.mode = 1;   // zero lag vector: every difference is 0, gamma stays 0
      G.mu = 1;
      G.ncta = 0;
    } else if (b == 0 && c == 0) {
      G.mode = 1;
      G.mu = std::max(1, a);
      G.mmax = nx;
      G.nqx = (ny + 31) / 32;   // row tiles
      G.nqb = nz;
      G.nmb = (nx + VT - 1) / VT;
      G.ncta = G.nmb * G.nqx * nz;
    } else {
      G.mode = 0;
      G.mu = 1;
      G.a = c != 0 ? 2 : 1;
      G.sig = c != 0 ? c : b;
      const int na = G.a == 2 ? nz : ny;
      const int sbv = G.a == 2 ? b : c;     // step of the other (y or z) axis
      const int nbv = G.a == 2 ? ny : nz;
      G.mmax = (na + G.sig - 1) / G.sig;
      const int mm1 = G.mmax - 1;
      long long qx_lo = -(long long)mm1 * std::max(a, 0), qx_hi = nx - 1 + (long long)mm1 * std::max(-a, 0);
      long long qb_lo = -(long long)mm1 * std::max(sbv, 0), qb_hi = nbv - 1 + (long long)mm1 * std::max(-sbv, 0);
      G.qx_lo = (int)qx_lo;
      G.nqx = (int)((qx_hi - qx_lo + 1 + 31) / 32);
      G.qb_lo = (int)qb_lo;
      G.nqb = (int)(qb_hi - qb_lo + 1);
      G.nmb = (G.mmax + VT - 1) / VT;
      long long ncta = (long long)G.nmb * G.nqx * G.nqb * G.sig;
      if (ncta > 0x7fffffffLL) {
        e = cudaErrorInvalidValue;
        break;
      }
      G.ncta = (int)ncta;
    }
    geos[d] = G;
    part_elems = std::max(part_elems, (size_t)G.ncta * VLCH);
  }
  // realizations per launch: partial buffer of at most 256 MB, grid.y <= 65535
  int rgroup = 1;
  if (part_elems) rgroup = (int)std::max<size_t>(1, ((size_t)256 << 20) / (part_elems * sizeof(double)));
  rgroup = std::min(std::min(rgroup, nreal), 65535);
  part_elems *= (size_t)rgroup;
  if (e == cudaSuccess && part_elems) e = cudaMalloc(&part, sizeof(double) * part_elems);
  for (int d = 0; d < ndir && e == cudaSuccess; d++) {
    const VarioGeo& G = geos[d];
    if (nlag[d] == 0 || G.ncta == 0) continue;
    // lag chunks: at most VLCH lags with nl * mu <= VPW (partner window bound)
    const int chunk = std::max(1, std::min(VLCH, VPW / std::max(1, G.mu)));
    for (int l0 = 1; l0 <= nlag[d] && e == cudaSuccess; l0 += chunk) {
      const int nl = std::min(chunk, nlag[d] - l0 + 1);
      const size_t smem = sizeof(double) * VP * (size_t)(VT + VT + (nl - 1) * G.mu);
      e = func_smem(reinterpret_cast<const void*>(k_vario), smem);
      if (e != cudaSuccess) break;
      std::vector<long long> npc(VLCH, 0);
      for (int li = 0; li < nl; li++) npc[li] = np_all[(l0 + li - 1) + (size_t)nlagmax * d];
      e = cudaMemcpyAsync(npdev, npc.data(), sizeof(long long) * VLCH, cudaMemcpyHostToDevice, st);
      for (int r0 = 0; r0 < nreal && e == cudaSuccess; r0 += rgroup) {
        const int nr = std::min(rgroup, nreal - r0);
        k_vario<<<dim3(G.ncta, nr), 32 * VNW, smem, st>>>(G, fdev + (size_t)r0 * M, (long long)M, l0, nl, part);
        ++g_launch_count;
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        k_vario_reduce<<<dim3(nl, nr), 256, 0, st>>>(part, G.ncta, l0, nl, d, ndir, nlagmax, npdev, gdev, r0);
        ++g_launch_count;
        e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // npdev is reused by the next chunk
    }
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(gam, gdev, sizeof(double) * ngam, dev_gam ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                        st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (fbuf) cudaFree(fbuf);
  if (gdev) cudaFree(gdev);
  if (part) cudaFree(part);
  if (npdev) cudaFree(npdev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(SS3D_ECUDA, (std::string("vario: ") + cudaGetErrorString(e)).c_str());
  }
  return SS3D_OK;
}
