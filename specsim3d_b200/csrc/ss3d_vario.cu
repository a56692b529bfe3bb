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
// Kernel layout.  Every direction is walked as lines with a unit march step:
//   * general (s has a y or z component): a line starts on one of the first
//     s_a planes of its leading axis a (z, else y) at a virtual start q that
//     may lie outside the grid, and steps by s; lanes of a CTA take 32
//     consecutive x starts (coalesced loads along each march step);
//   * pure x (s = (sx, 0, 0)): a line is row (y, z) restricted to the
//     residue x = rho (mod sx), rho < min(sx, nx); lanes take 32 rows.
// Each lane's line meets the grid on one interval of march indices; the lane
// counts its march from the first point inside (lane-local index), so a pair
// (base b, partner b + l) is valid iff the partner index is below the lane's
// line length.  A CTA owns the lane-local bases [m0, m0 + Tb) of its 32 lines
// and stages their values in shared memory s[row][lane] (pitch 33 doubles).
// Warp w owns the lags l0 + 16 w + j (j < 16) of the launch and runs register
// blocks of 8 bases x 16 lags: 8 base values and 23 partner values serve 128
// pairs, one FP64 subtraction and one FP64 fma per pair.  Lane sums are
// folded per lag in a fixed order and written as per-CTA partials, reduced by
// k_vario_reduce in CTA order: results do not depend on scheduling.
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

constexpr int VT = 256;            // lane-local bases per CTA at most
constexpr int VB = 8;              // bases per register block
constexpr int VL = 16;             // lags per warp
constexpr int VNW = 8;             // warps per CTA at most
constexpr int VLCH = VNW * VL;     // lags per launch (128)
constexpr int VP = 33;             // shared-memory pitch (lanes + 1)
static_assert(VT % VB == 0, "a CTA's base range is a whole number of register blocks");

struct VarioGeo {
  int nx, ny, nz;
  int mode;          // 0 general, 1 pure x
  int sx, sy, sz;    // normalised direction
  int a;             // general: leading axis 1 = y, 2 = z
  int sig;           // general: s_a > 0; pure x: residues min(sx, nx)
  int qx_lo, nqx;    // general: virtual start range along x (32 per tile); pure x: row tiles
  int qb_lo, nqb;    // general: virtual start range along the other axis; pure x: planes
  int mmax;          // longest line (march steps inside the grid)
  int tb;            // lane-local bases per CTA (multiple of VB)
  int nmb;           // base blocks of tb per line
  int ncta;          // CTAs per realization
};

// Launch layout of one lag chunk: shared rows [0, na) hold lane-local march
// m0 .. m0 + na - 1; rows [na, na + nb) (split layout) hold m0 + l0 .. ;
// the partner of base row b at lag l0 + k sits at row pofs + b + k, and is
// staged when b + k < prow.
struct VarioWin {
  int l0, nl;        // lags l0 .. l0 + nl - 1
  int na, nb;        // staged rows of the two segments (nb = 0: one segment)
  int pofs, prow;    // partner row of (b, k = 0) and the partner rows staged
  int rows;          // rows allocated (na + nb + VB: base blocks may read past)
};

__host__ __device__ __forceinline__ long long floordiv(long long a, long long b) {  // b > 0
  return a >= 0 ? a / b : -((-a + b - 1) / b);
}
__host__ __device__ __forceinline__ long long ceildiv(long long a, long long b) { return -floordiv(-a, b); }

// Line of lane t of CTA cta: linear index of its first point inside the grid
// (base), linear step, number of points inside (len) and the first lane-local
// base m0 of the CTA.
__device__ __forceinline__ void lane_line(const VarioGeo& G, int cta, int t, int& len, long long& base,
                                          long long& step, int& m0) {
  const int mb = cta % G.nmb;
  int rest = cta / G.nmb;
  m0 = mb * G.tb;
  long long x0, y0, z0, dx, dy, dz;
  long long hi = G.mmax;
  if (G.mode == 1) {
    const int jt = rest % G.nqx;
    rest /= G.nqx;
    const int k = rest % G.nqb;
    const int rho = rest / G.nqb;
    x0 = rho;
    y0 = (long long)jt * 32 + t;
    z0 = k;
    dx = G.sx;
    dy = 0;
    dz = 0;
  } else {
    const int xt = rest % G.nqx;
    rest /= G.nqx;
    const int qb = G.qb_lo + rest % G.nqb;
    const int r = rest / G.nqb;
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
  long long lo = 0;
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
  len = (int)(hi - lo);
  step = dx + (long long)G.nx * (dy + (long long)G.ny * dz);
  // first point inside; for an empty line any in-range index (never read)
  base = len > 0 ? x0 + (long long)G.nx * (y0 + (long long)G.ny * z0) + lo * step : 0;
}

__device__ __forceinline__ double vload(const double* __restrict__ fr, long long base, long long step, int m,
                                        int len) {
  return m < len ? __ldg(fr + base + (long long)m * step) : 0.0;
}

__global__ void __launch_bounds__(32 * VNW, 3) k_vario(VarioGeo G, VarioWin W, const double* __restrict__ f,
                                                    long long fstride, double* __restrict__ part) {
  extern __shared__ __align__(16) double smv[];
  const int r = blockIdx.y;
  const int cta = blockIdx.x;
  const int t = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const double* fr = f + (long long)r * fstride;
  int len, m0;
  long long base, step;
  lane_line(G, cta, t, len, base, step, m0);
  // ---- staging: segment A march m0 + q -> row q; segment B march m0 + l0 + q -> row na + q;
  // the VB rows past them are zero (read by the last base block, never used)
  const int nrow = W.na + W.nb;
  if (G.mode == 0) {
    for (int q = w; q < W.rows; q += nw) {
      double v = 0.0;
      if (q < W.na)
        v = vload(fr, base, step, m0 + q, len);
      else if (q < nrow)
        v = vload(fr, base, step, m0 + W.l0 + (q - W.na), len);
      smv[q * VP + t] = v;
    }
  } else {
    for (int row = w; row < 32; row += nw) {
      int rlen, rm0;
      long long rbase, rstep;
      lane_line(G, cta, row, rlen, rbase, rstep, rm0);
      for (int q = t; q < W.rows; q += 32) {
        double v = 0.0;
        if (q < W.na)
          v = vload(fr, rbase, rstep, m0 + q, rlen);
        else if (q < nrow)
          v = vload(fr, rbase, rstep, m0 + W.l0 + (q - W.na), rlen);
        smv[q * VP + row] = v;
      }
    }
  }
  __syncthreads();
  // ---- pairs: bases b in [0, tb), lags l0 + lw + j; partner row pofs + b + lw + j,
  // valid while b + lw + j < plim (inside the line and inside the staged rows)
  const int lw = w * VL;
  const int plim = min(len - m0 - W.l0, W.prow);
  const int bmax = min(G.tb, __reduce_max_sync(0xffffffffu, plim) - lw);
  double acc[VL];
#pragma unroll
  for (int j = 0; j < VL; ++j) acc[j] = 0.0;
  const double* sl = smv + t;
  for (int b0 = 0; b0 < bmax; b0 += VB) {
    double bv[VB];
#pragma unroll
    for (int i = 0; i < VB; ++i) bv[i] = sl[(b0 + i) * VP];
    const int q0 = b0 + lw;
    const double* pp = sl + (W.pofs + q0) * VP;
#pragma unroll
    for (int p = 0; p < VB + VL - 1; ++p) {
      if (q0 + p < plim) {
        const double pv = pp[p * VP];
#pragma unroll
        for (int i = (p - VL + 1 > 0 ? p - VL + 1 : 0); i <= (p < VB - 1 ? p : VB - 1); ++i) {
          const double d = pv - bv[i];
          acc[p - i] = fma(d, d, acc[p - i]);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < VL; ++j) {
    double v = acc[j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (t == 0 && lw + j < W.nl) part[((long long)r * G.ncta + cta) * VLCH + lw + j] = v;
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

const void* module_anchor_vario() { return reinterpret_cast<const void*>(k_vario_reduce); }

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
    e = cudaMallocAsync((void**)&fbuf, sizeof(double) * M * nreal, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(fbuf, res, sizeof(double) * M * nreal, cudaMemcpyHostToDevice, st);
    fdev = fbuf;
  }
  // temporaries from the stream-ordered pool: no device-wide synchronisation
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&gdev, sizeof(double) * ngam, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(gdev, 0, sizeof(double) * ngam, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&npdev, sizeof(long long) * VLCH, st);
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
    long long ncta = 0;
    if (a == 0 && b == 0 && c == 0) {
      G.mode = 1;   // zero lag vector: every difference is 0, gamma stays 0
    } else if (b == 0 && c == 0) {
      G.mode = 1;
      G.sig = std::min(a, nx);                // residues rho < min(sx, nx)
      G.mmax = (nx + a - 1) / a;
      G.nqx = (ny + 31) / 32;                 // row tiles
      G.nqb = nz;
      ncta = (long long)G.nqx * nz * G.sig;
    } else {
      G.mode = 0;
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
      ncta = (long long)G.nqx * G.nqb * G.sig;
    }
    if (ncta > 0) {
      G.tb = std::min(VT, (G.mmax + VB - 1) / VB * VB);
      G.nmb = (G.mmax + G.tb - 1) / G.tb;
      ncta *= G.nmb;
    }
    if (ncta > 0x7fffffffLL) {
      e = cudaErrorInvalidValue;
      break;
    }
    G.ncta = (int)ncta;
    geos[d] = G;
    part_elems = std::max(part_elems, (size_t)G.ncta * VLCH);
  }
  // realizations per launch: partial buffer of at most 256 MB, grid.y <= 65535
  int rgroup = 1;
  if (part_elems) rgroup = (int)std::max<size_t>(1, ((size_t)256 << 20) / (part_elems * sizeof(double)));
  rgroup = std::min(std::min(rgroup, nreal), 65535);
  part_elems *= (size_t)rgroup;
  if (e == cudaSuccess && part_elems) e = cudaMallocAsync((void**)&part, sizeof(double) * part_elems, st);
  for (int d = 0; d < ndir && e == cudaSuccess; d++) {
    const VarioGeo& G = geos[d];
    if (nlag[d] == 0 || G.ncta == 0) continue;
    for (int l0 = 1; l0 <= nlag[d] && e == cudaSuccess; l0 += VLCH) {
      VarioWin W{};
      W.l0 = l0;
      W.nl = std::min(VLCH, nlag[d] - l0 + 1);
      const int nw = (W.nl + VL - 1) / VL;
      // partners of base b < tb at lag offsets k < nw VL lie at lane-local
      // march m0 + l0 + b + k; march steps past the longest line are never read
      const int span = std::min(G.tb + nw * VL - 1, std::max(0, G.mmax - l0));
      const int one = std::min(G.mmax, l0 + span);   // rows of one segment from m0
      if (one <= G.tb + span) {
        W.na = one;
        W.nb = 0;
        W.pofs = l0;
        W.prow = std::max(0, one - l0);
      } else {
        W.na = G.tb;
        W.nb = span;
        W.pofs = G.tb;
        W.prow = span;
      }
      W.rows = W.na + W.nb + VB;
      const size_t smem = sizeof(double) * VP * (size_t)W.rows;
      e = func_smem(reinterpret_cast<const void*>(k_vario), smem);
      if (e != cudaSuccess) break;
      std::vector<long long> npc(VLCH, 0);
      for (int li = 0; li < W.nl; li++) npc[li] = np_all[(l0 + li - 1) + (size_t)nlagmax * d];
      e = cudaMemcpyAsync(npdev, npc.data(), sizeof(long long) * VLCH, cudaMemcpyHostToDevice, st);
      for (int r0 = 0; r0 < nreal && e == cudaSuccess; r0 += rgroup) {
        const int nr = std::min(rgroup, nreal - r0);
        k_vario<<<dim3(G.ncta, nr), 32 * nw, smem, st>>>(G, W, fdev + (size_t)r0 * M, (long long)M, part);
        ++g_launch_count;
        e = cudaGetLastError();
        if (e != cudaSuccess) break;
        k_vario_reduce<<<dim3(W.nl, nr), 256, 0, st>>>(part, G.ncta, l0, W.nl, d, ndir, nlagmax, npdev, gdev, r0);
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
  if (fbuf) cudaFreeAsync(fbuf, st);
  if (gdev) cudaFreeAsync(gdev, st);
  if (part) cudaFreeAsync(part, st);
  if (npdev) cudaFreeAsync(npdev, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(SS3D_ECUDA, (std::string("vario: ") + cudaGetErrorString(e)).c_str());
  }
  return SS3D_OK;
}
