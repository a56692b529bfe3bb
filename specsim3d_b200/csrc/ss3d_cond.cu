// ss3d_cond.cu -- conditioning by kriging of the residual
// (reference: condition_field f90:700-1081, nscore/backtr/gauinv f90:557-697).
//
//   z_c(x) = z*_SK(x; data) + [ z_s(x) - z*_SK(x; z_s at the data nodes) ]
//
// Host (small, serial in the reference too): data snapping and trimming,
// merging of data that share a node (heapsort order, weighted mean), normal
// scores, super-block tables.  GPU: the neighbour search of every node
// (thread per node), the simple-kriging solve of every node (warp per node,
// matrix in shared memory), the back transform (thread per cell).
//
// The search reproduces the reference's neighbour set exactly: squared scaled
// distances are formed with round-to-nearest intrinsics in the reference's
// expression order (no FMA contraction), blocks are visited in the same
// kb, jb, ib order, data inside a block in index order, and the list keeps
// the ndmax smallest with the same insertion rules (strict < to replace the
// last entry when full, insertion after equal distances).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/specsim3d_gpu.h"
#include "ss3d_internal.h"

namespace ss3d {

// Leading dimension of the kriging matrices in shared memory: odd, so that the
// lanes of a warp walking down a column (stride ld elements) hit distinct banks
// (an even ld such as ndmax = 24 put 16 lanes on the same bank pair).
__host__ __device__ inline int cond_ld(int ndmax) { return ndmax | 1; }

// shared memory of one kriging warp.  FP64 solves (prec 0): the covariance
// matrix with the right-hand side as an extra row, factored in place
// ((ndmax + 1) x ld doubles), four ndmax vectors of doubles and the neighbour
// ids.  FP32 solves (prec 1): the FP64 matrix (kept for the refinement
// residual), its FP32 factor with the extra row ((ndmax + 1) x ld floats),
// three ndmax vectors of doubles, four of floats and the ids.  Rounded up to 16
// bytes.
__host__ __device__ inline size_t cond_warp_bytes(int ndmax, int prec) {
  const size_t n = (size_t)ndmax, m = (n + 1) * (size_t)cond_ld(ndmax);
  const size_t b = (prec == 0 ? m * 8 + n * 32 + n * 4 : m * 12 + n * 24 + n * 16 + n * 4) + n * 12;
  return (b + 15) & ~(size_t)15;
}

struct CondGeo {
  int nx, ny, nz, nreal, nd, ndmax;
  double xmin, ymin, zmin, dx, dy, dz;
  int nsbx, nsby, nsbz, mbx, mby, mbz;
  double bsx, bsy, bsz;
  double rot[9];       // search ellipsoid rotation (setrot of the search "structure")
  double rmax2;        // rmax * rmax
  double c0;           // C(0)
  int nrow;            // rows of super-block offsets in the scan list
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// The covariance model of the kriging systems (f90:153-178) with each
// structure's rotation divided by its range, so that h / a takes no division
// per evaluation; the same value as covariance() up to the rounding of the
// scaled rotation.
struct KModel {
  int nst;
  double nugget;
  int itype[MAXST];
  double sill[MAXST];
  double rots[MAXST][9];
};
__device__ __forceinline__ double cov_k(const KModel& m, double dx, double dy, double dz) {
  double c = (dx == 0.0 && dy == 0.0 && dz == 0.0) ? m.nugget : 0.0;
  for (int i = 0; i < m.nst; i++) {
    const double* r = m.rots[i];
    const double rx = r[0] * dx + r[1] * dy + r[2] * dz;
    const double ry = r[3] * dx + r[4] * dy + r[5] * dz;
    const double rz = r[6] * dx + r[7] * dy + r[8] * dz;
    const double hr = sqrt(rx * rx + ry * ry + rz * rz);
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

// Covariance of integer lattice lags.  Data are snapped to nodes (f90:789-792,
// 826), so every entry of a kriging system is C(di dx, dj dy, dk dz) for an
// integer lag (di, dj, dk): the difference of two data nodes or of a data node
// and the node kriged.  Both lie inside the search ellipsoid around the node,
// so |di| <= 2 e_x / dx (e_x the half-extent of the ellipsoid along x), and so
// on.  The table holds C over that box for dk >= 0 (C(-h) = C(h)), built once
// per call; a lag outside it (or no table, when the box is too large) is
// evaluated directly.
struct CovTab {
  const double* v;   // [dk][dj + ty][di + tx], dk in [0, tz]; NULL: no table
  int tx, ty, tz;
};
__device__ __forceinline__ double cov_lat(const CovTab& T, const KModel& m, int di, int dj, int dk, double dx,
                                          double dy, double dz) {
  if (dk < 0) {
    di = -di;
    dj = -dj;
    dk = -dk;
  }
  if (T.v && dk <= T.tz && abs(dj) <= T.ty && abs(di) <= T.tx)
    return __ldg(T.v + (di + T.tx) + (size_t)(2 * T.tx + 1) * ((dj + T.ty) + (size_t)(2 * T.ty + 1) * dk));
  return cov_k(m, (double)di * dx, (double)dj * dy, (double)dk * dz);
}

// the same lookup with the out-of-table case as a call on a model in global
// memory (keeps the kernels that unroll their fills small)
__device__ __noinline__ double cov_lag_direct(const KModel* __restrict__ m, int di, int dj, int dk, double dx,
                                              double dy, double dz) {
  return cov_k(*m, (double)di * dx, (double)dj * dy, (double)dk * dz);
}
__device__ __forceinline__ double cov_lat_g(const CovTab& T, const KModel* __restrict__ m, int di, int dj, int dk,
                                            double dx, double dy, double dz) {
  if (dk < 0) {
    di = -di;
    dj = -dj;
    dk = -dk;
  }
  if (T.v && dk <= T.tz && abs(dj) <= T.ty && abs(di) <= T.tx)
    return __ldg(T.v + (di + T.tx) + (size_t)(2 * T.tx + 1) * ((dj + T.ty) + (size_t)(2 * T.ty + 1) * dk));
  return cov_lag_direct(m, di, dj, dk, dx, dy, dz);
}

__global__ void k_cov_table(KModel m, double dx, double dy, double dz, int tx, int ty, int tz, double* __restrict__ v) {
  const long long wx = 2 * tx + 1, wy = 2 * ty + 1, tot = wx * wy * (tz + 1);
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int di = (int)(q % wx) - tx;
    const int dj = (int)((q / wx) % wy) - ty;
    const int dk = (int)(q / (wx * wy));
    v[q] = cov_k(m, (double)di * dx, (double)dj * dy, (double)dk * dz);
  }
}

// 1/sqrt(x) for a positive normal x: the hardware approximation (PTX
// rsqrt.approx) refined by Newton's iteration r <- r + r (1 - x r^2) / 2,
// twice in FP64 (about 2^-23 -> 2^-46 -> full precision) and once in FP32.
__device__ __forceinline__ double rsqrt_nr(double x) {
  double r;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x * r, r, 1.0);
  r = fma(0.5 * r, e, r);
  e = fma(-x * r, r, 1.0);
  return fma(0.5 * r, e, r);
}
__device__ __forceinline__ float rsqrt_nr(float x) {
  float r;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  const float e = fmaf(-x * r, r, 1.0f);
  return fmaf(0.5f * r, e, r);
}

// neighbour search of nodes [node0, node0 + count): writes nn and the
// neighbour ids (0-based data index) and flags the exact data nodes.
// sxyz[p] = (x, y, z, id) of the p-th datum in super-block order (the order of
// sbidx), so that the scan of a super block reads its data directly.  The
// candidate list of a thread (CAP >= ndmax entries) lives in shared memory,
// entry m of thread t at [m][t]; BS threads per block keep it within the
// 48 KB of static shared memory.
// A candidate is rejected when s = rx^2 + ry^2 + rz^2 > rmax^2, with no
// division: for correctly rounded division RN(s / c) > 1 holds exactly when
// s > c (s > c means s >= c + ulp(c), so s / c > 1 + 2^-53, above the midpoint
// between 1 and its successor), so the test is the reference's d2 > 1
// (f90:1249-1262); accepted candidates get d2 = RN(s / rmax^2) as there.
// rows[r] = (x offset from, x offset to, y offset, z offset): the super-block
// offsets of the search box by rows along x, in the reference's scan order (z,
// then y, then x block ascending), without the blocks that can hold no datum
// inside the ellipsoid for any node of the centre block (super_block_rows):
// their candidates would all be rejected, so the kept neighbours and their
// order are the same.  The data of the blocks of one row are contiguous in
// super-block order, so a row is one range of sxyz.
template <int CAP> struct SearchCfg {
  static constexpr int BS = CAP <= 32 ? 128 : (CAP <= 64 ? 64 : 32);
};
template <int CAP>
__global__ void __launch_bounds__(SearchCfg<CAP>::BS) k_cond_search(CondGeo G, long long node0, int count,
                                                                   const double4* __restrict__ sxyz,
                                                                   const int* __restrict__ sbstart,
                                                                   const int4* __restrict__ rows,
                                                                   const int* __restrict__ ix,
                                                                   const int* __restrict__ iy,
                                                                   const int* __restrict__ iz, int* __restrict__ nbr,
                                                                   int* __restrict__ nnb) {
  constexpr int BS = SearchCfg<CAP>::BS;
  __shared__ double cds[CAP][BS];
  __shared__ int cids[CAP][BS];
  const int t = threadIdx.x;
  const int q = blockIdx.x * BS + t;
  if (q >= count) return;
  const long long node = node0 + q;
  const int i = (int)(node % G.nx) + 1;
  const int j = (int)((node / G.nx) % G.ny) + 1;
  const int k = (int)(node / ((long long)G.nx * G.ny)) + 1;
  const double x = __dadd_rn(G.xmin, __dmul_rn((double)(i - 1), G.dx));
  const double y = __dadd_rn(G.ymin, __dmul_rn((double)(j - 1), G.dy));
  const double z = __dadd_rn(G.zmin, __dmul_rn((double)(k - 1), G.dz));
  const int bx = clampi((int)__ddiv_rn(__dadd_rn(__dsub_rn(x, G.xmin), __dmul_rn(0.5, G.dx)), G.bsx) + 1, 1, G.nsbx);
  const int by = clampi((int)__ddiv_rn(__dadd_rn(__dsub_rn(y, G.ymin), __dmul_rn(0.5, G.dy)), G.bsy) + 1, 1, G.nsby);
  const int bz = clampi((int)__ddiv_rn(__dadd_rn(__dsub_rn(z, G.zmin), __dmul_rn(0.5, G.dz)), G.bsz) + 1, 1, G.nsbz);
  int nn = 0;
  const int ndmax = G.ndmax;
  double worst = 0.0;   // cds[nn - 1][t] once the list is full
  const double r0 = G.rot[0], r1 = G.rot[1], r2 = G.rot[2], r3 = G.rot[3], r4 = G.rot[4], r5 = G.rot[5],
               r6 = G.rot[6], r7 = G.rot[7], r8 = G.rot[8], rmax2 = G.rmax2;
  for (int o = 0; o < G.nrow; ++o) {
    const int4 rw = __ldg(rows + o);
    const int jb = by + rw.z, kb = bz + rw.w;
    const int ib0 = max(1, bx + rw.x), ib1 = min(G.nsbx, bx + rw.y);
    if (jb < 1 || jb > G.nsby || kb < 1 || kb > G.nsbz || ib0 > ib1) continue;
    const int row0 = G.nsbx * (jb - 1 + G.nsby * (kb - 1));
    const int p1 = __ldg(sbstart + row0 + ib1) - 1;
    for (int p = __ldg(sbstart + row0 + ib0 - 1); p <= p1; ++p) {
      const double2 a = __ldg(reinterpret_cast<const double2*>(sxyz + p - 1));
      const double2 b = __ldg(reinterpret_cast<const double2*>(sxyz + p - 1) + 1);
      const double hx = __dsub_rn(a.x, x), hy = __dsub_rn(a.y, y), hz = __dsub_rn(b.x, z);
      const double rx = __dadd_rn(__dadd_rn(__dmul_rn(r0, hx), __dmul_rn(r1, hy)), __dmul_rn(r2, hz));
      const double ry = __dadd_rn(__dadd_rn(__dmul_rn(r3, hx), __dmul_rn(r4, hy)), __dmul_rn(r5, hz));
      const double rz = __dadd_rn(__dadd_rn(__dmul_rn(r6, hx), __dmul_rn(r7, hy)), __dmul_rn(r8, hz));
      const double s2 = __dadd_rn(__dadd_rn(__dmul_rn(rx, rx), __dmul_rn(ry, ry)), __dmul_rn(rz, rz));
      if (s2 > rmax2) continue;
      const double d2 = __ddiv_rn(s2, rmax2);
      int m;
      if (nn < ndmax) {
        nn = nn + 1;
        m = nn;
      } else if (d2 < worst) {
        m = nn;
      } else {
        continue;
      }
      while (m > 1) {
        const double prev = cds[m - 2][t];
        if (prev <= d2) break;
        cds[m - 1][t] = prev;
        cids[m - 1][t] = cids[m - 2][t];
        m = m - 1;
      }
      cds[m - 1][t] = d2;
      cids[m - 1][t] = (int)b.y;
      if (nn == ndmax) worst = cds[nn - 1][t];
    }
  }
  int* out = nbr + (long long)q * ndmax;
  for (int m = 0; m < nn; ++m) out[m] = cids[m][t];
  // exact data node: nearest at distance 0 and on this very node
  int flag = 0;
  if (nn > 0 && cds[0][t] == 0.0) {
    const int d = cids[0][t];
    if (__ldg(ix + d) == i && __ldg(iy + d) == j && __ldg(iz + d) == k) flag = 1;
  }
  nnb[q] = nn | (flag << 16);
}

// Lower-triangle pair table shared by a block: entry e (row-major over the
// lower triangle with the diagonal) holds (r, c), c <= r, in two bytes, so that
// the lanes of a warp can take the elements of a triangle in turn without a
// division.  Entries of a triangle of side m are the first m (m + 1) / 2.
__host__ __device__ inline size_t cond_tri_bytes(int ndmax) {
  return ((size_t)ndmax * (ndmax + 1) / 2 * 2 + 15) & ~(size_t)15;
}

__device__ inline void fill_tri(uint8_t* tri, int ndmax) {
  const int T = ndmax * (ndmax + 1) / 2;
  for (int e = threadIdx.x; e < T; e += blockDim.x) {
    int r = (int)((sqrtf(8.0f * (float)e + 1.0f) - 1.0f) * 0.5f);
    while (r * (r + 1) / 2 > e) --r;
    while ((r + 1) * (r + 2) / 2 <= e) ++r;
    tri[2 * e] = (uint8_t)r;
    tri[2 * e + 1] = (uint8_t)(e - r * (r + 1) / 2);
  }
}

// Forward and back substitution with the factor L (lower, leading dimension
// ld) whose diagonal reciprocals are rinv: L L^T w = b, warp-parallel by
// columns; tmp is n scratch values.
template <typename T>
__device__ void warp_tri_solve(const T* L, const T* rinv, int ld, int n, T* w, const T* b, T* tmp, int lane) {
  for (int p = lane; p < n; p += 32) tmp[p] = b[p];
  __syncwarp();
  for (int p = 0; p < n; ++p) {
    const T wp = tmp[p] * rinv[p];
    for (int r = p + 1 + lane; r < n; r += 32) tmp[r] -= L[r * ld + p] * wp;
    if (lane == 0) w[p] = wp;
    __syncwarp();
  }
  for (int p = lane; p < n; p += 32) tmp[p] = w[p];
  __syncwarp();
  for (int p = n - 1; p >= 0; --p) {
    const T wp = tmp[p] * rinv[p];
    for (int r = lane; r < p; r += 32) tmp[r] -= L[p * ld + r] * wp;
    if (lane == 0) w[p] = wp;
    __syncwarp();
  }
}

// back substitution L^T w = y with the factor L (diagonal reciprocals rinv);
// tmp is n scratch values
template <typename T>
__device__ void warp_tri_back(const T* L, const T* rinv, int ld, int n, T* w, const T* y, T* tmp, int lane) {
  for (int p = lane; p < n; p += 32) tmp[p] = y[p];
  __syncwarp();
  for (int p = n - 1; p >= 0; --p) {
    const T wp = tmp[p] * rinv[p];
    for (int r = lane; r < p; r += 32) tmp[r] -= L[p * ld + r] * wp;
    if (lane == 0) w[p] = wp;
    __syncwarp();
  }
}

// Cholesky factor of L + ridge I in place (lower triangle; L holds the matrix
// on entry), warp-cooperative and right-looking: the trailing update of each
// column goes over the lanes by the pair table (each element receives its
// updates in column order, as in the serial algorithm); the column is scaled
// by the reciprocal of its pivot, kept in rinv for the solves.  Row n holds a
// right-hand side b and is carried through the same scalings and updates, so
// that it ends as y = L^-1 b, the forward substitution done on the way.
// Returns false on a non-positive pivot (the reference's chol_solve failure,
// f90:1040-1079).
template <typename T>
__device__ bool warp_cholesky(T* L, T* rinv, int ld, int n, T ridge, const uint8_t* __restrict__ tri, int lane) {
  for (int p = lane; p < n; p += 32) L[p * ld + p] += ridge;
  __syncwarp();
  T* y = L + (size_t)n * ld;
  for (int c = 0; c < n; ++c) {
    const T piv = L[c * ld + c];
    if (!(piv > T(0))) return false;   // uniform: every lane reads the same value
    const T inv = rsqrt_nr(piv);       // 1 / sqrt(pivot)
    const T dgl = piv * inv;
    __syncwarp();
    for (int r = c + 1 + lane; r <= n; r += 32) L[r * ld + c] *= inv;   // row n: y_c
    if (lane == 0) {
      L[c * ld + c] = dgl;
      rinv[c] = inv;
    }
    __syncwarp();
    const int m = n - c - 1, nt = m * (m + 1) / 2;
    for (int e = lane; e < nt; e += 32) {
      const int r = c + 1 + tri[2 * e], cc = c + 1 + tri[2 * e + 1];
      L[r * ld + cc] -= L[r * ld + c] * L[cc * ld + c];
    }
    for (int cc = c + 1 + lane; cc < n; cc += 32) y[cc] -= y[c] * L[cc * ld + c];
    __syncwarp();
  }
  return true;
}

// kriging of the residual at nodes [node0, node0+count): warp per node.
// precision 0: FP64 factor and solve; 1: FP32 factor and solve plus one
// refinement step with the residual b - A w formed in FP64.
// Dynamic shared memory: the pair table, then one region per warp.
template <int PREC>
__global__ void k_cond_krige(CondGeo G, KModel mdl, CovTab ctab, long long node0, int count,
                             const int* __restrict__ nbr, const int* __restrict__ nnb, const int* __restrict__ ixs,
                             const int* __restrict__ iys, const int* __restrict__ izs,
                             const double* __restrict__ dg, const double* __restrict__ simd, double* __restrict__ res,
                             unsigned long long* __restrict__ counters) {
  extern __shared__ __align__(16) unsigned char smc[];
  __shared__ unsigned long long bcount[4];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwb = blockDim.x >> 5;
  const int ndmax = G.ndmax;
  const int ld = cond_ld(ndmax);
  uint8_t* tri = smc;
  fill_tri(tri, ndmax);
  if (threadIdx.x < 4) bcount[threadIdx.x] = 0;
  __syncthreads();
  const size_t per = cond_warp_bytes(ndmax, PREC);
  unsigned char* mine = smc + cond_tri_bytes(ndmax) + per * wib;
  const int n2 = (ndmax + 1) * ld;   // matrix rows and the right-hand-side row
  double* A = (double*)mine;     // covariance matrix (PREC 0: factored in place)
  double* b = A + n2;
  double* w = b + ndmax;
  double* tmp = w + ndmax;
  double* rinv = tmp + ndmax;    // PREC 0 only
  float* Lf = (float*)(tmp + ndmax);   // PREC 1: FP32 factor, then bf, wf, tf, rinvf
  float* bf = Lf + n2;
  float* wf = bf + ndmax;
  float* tf = wf + ndmax;
  float* rinvf = tf + ndmax;
  int* id = PREC == 0 ? (int*)(rinv + ndmax) : (int*)(rinvf + ndmax);
  int* lat = id + ndmax;         // lattice indices (0-based) of the neighbours: x, y, z per neighbour
  const long long M = (long long)G.nx * G.ny * G.nz;
  for (int q = blockIdx.x * nwb + wib; q < count; q += gridDim.x * nwb) {
    const long long node = node0 + q;
    const int code = nnb[q];
    const int nn = code & 0xffff, exact = code >> 16;
    if (lane == 0) atomicAdd_block(&bcount[0], (unsigned long long)nn);
    if (nn == 0) {
      if (lane == 0) atomicAdd_block(&bcount[2], 1ull);
      continue;
    }
    const int* nl = nbr + (long long)q * ndmax;
    if (exact) {
      const double v = dg[nl[0]];
      for (int l = lane; l < G.nreal; l += 32) res[node + M * l] = v;
      if (lane == 0) atomicAdd_block(&bcount[3], 1ull);
      continue;
    }
    // a conditioned grid has at most 2^27 nodes: 32-bit index arithmetic
    const uint32_t nu = (uint32_t)node, row = nu / (uint32_t)G.nx;
    const int i = (int)(nu - row * (uint32_t)G.nx), j = (int)(row % (uint32_t)G.ny), k = (int)(row / (uint32_t)G.ny);
    for (int p = lane; p < nn; p += 32) {
      const int cp = nl[p];
      id[p] = cp;
      lat[3 * p] = __ldg(ixs + cp) - 1;
      lat[3 * p + 1] = __ldg(iys + cp) - 1;
      lat[3 * p + 2] = __ldg(izs + cp) - 1;
    }
    __syncwarp();
    const int ntri = nn * (nn + 1) / 2;
    auto fill_matrix = [&]() {
      for (int e = lane; e < ntri; e += 32) {
        const int p = tri[2 * e], qq = tri[2 * e + 1];
        const double v = cov_lat(ctab, mdl, lat[3 * p] - lat[3 * qq], lat[3 * p + 1] - lat[3 * qq + 1],
                                 lat[3 * p + 2] - lat[3 * qq + 2], G.dx, G.dy, G.dz);
        A[p * ld + qq] = v;
        A[qq * ld + p] = v;
      }
    };
    fill_matrix();
    for (int p = lane; p < nn; p += 32)
      b[p] = cov_lat(ctab, mdl, lat[3 * p] - i, lat[3 * p + 1] - j, lat[3 * p + 2] - k, G.dx, G.dy, G.dz);
    __syncwarp();
    double ridge = 1.0e-10 * G.c0;
    bool ok = false;
    int tries = 0;
    for (tries = 1; tries <= 3; ++tries) {
      if (PREC == 0) {
        if (tries > 1) {   // the failed factorization overwrote the matrix
          fill_matrix();
        }
        for (int p = lane; p < nn; p += 32) A[nn * ld + p] = b[p];   // right-hand side row
        __syncwarp();
        ok = warp_cholesky<double>(A, rinv, ld, nn, ridge, tri, lane);
        if (ok) warp_tri_back<double>(A, rinv, ld, nn, w, A + nn * ld, tmp, lane);
      } else {
        // FP32 copies of A and b; the factor is built in place in Lf, b as its row nn
        for (int e = lane; e < nn * ld; e += 32) Lf[e] = (float)A[e];
        for (int p = lane; p < nn; p += 32) Lf[nn * ld + p] = (float)b[p];
        __syncwarp();
        ok = warp_cholesky<float>(Lf, rinvf, ld, nn, (float)ridge, tri, lane);
        if (ok) {
          warp_tri_back<float>(Lf, rinvf, ld, nn, wf, Lf + nn * ld, tf, lane);
          // one refinement: res = b - (A + ridge I) w in FP64 (to tmp), solve
          // L L^T d = res in FP32, w += d
          for (int p = lane; p < nn; p += 32) w[p] = (double)wf[p];
          __syncwarp();
          for (int p = lane; p < nn; p += 32) {
            double sres = b[p] - ridge * w[p];
            for (int m = 0; m < nn; ++m) sres -= A[p * ld + m] * w[m];
            tmp[p] = sres;
          }
          __syncwarp();
          for (int p = lane; p < nn; p += 32) bf[p] = (float)tmp[p];
          __syncwarp();
          warp_tri_solve<float>(Lf, rinvf, ld, nn, wf, bf, tf, lane);
          for (int p = lane; p < nn; p += 32) w[p] += (double)wf[p];
          __syncwarp();
        }
      }
      if (ok) break;
      ridge = ridge * 1.0e3;
    }
    if (!ok) {
      if (lane == 0) atomicAdd_block(&bcount[1], 1ull);
      continue;
    }
    if (tries > 1 && lane == 0) atomicAdd_block(&bcount[1], 1ull);
    double zk = 0.0;   // sum of w dg over the neighbours: lanes, then a butterfly
    for (int p = lane; p < nn; p += 32) zk += w[p] * dg[id[p]];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) zk += __shfl_xor_sync(0xffffffffu, zk, off);
    for (int l = lane; l < G.nreal; l += 32) {
      double sks = 0.0;
      for (int p = 0; p < nn; ++p) sks += w[p] * simd[(long long)id[p] * G.nreal + l];
      res[node + M * l] = zk + res[node + M * l] - sks;
    }
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x < 4 && bcount[threadIdx.x]) atomicAdd(&counters[threadIdx.x], bcount[threadIdx.x]);
}

// GSLIB back transform (backtr, powint, gcum), f90:628-697, of one value.
// mode 0: none; 1: back transform through the normal-score table (gt, vr),
// itrans 1; 2: add the simple-kriging mean (itrans 0, skmean != 0).  The
// bracket gt[lo-1] <= y < gt[lo] of the table's bisection is the count of
// entries <= y; it is found from a bucket index (base[k] = entries <= gt[0] +
// k w) and corrected by steps along the table, so it is exactly the
// bisection's whatever bucket the rounding of k picks.
struct BackTr {
  const double* vr;
  const double* gt;
  const int* base;   // nbucket + 1 counts; NULL: bisection
  int nt, nbucket, mode, lt, ut;
  double zmin, zmax, ltp, utp, skmean, g0, inv_w;
};
__device__ __forceinline__ double powint_d(double xlow, double xhigh, double ylow, double yhigh, double xval, double pw) {
  if (xhigh - xlow < 1.0e-20) return 0.5 * (ylow + yhigh);
  // t^1 = t exactly (the value a correctly rounded pow returns): the linear
  // interpolation between table entries, the common case, takes no pow
  const double t = (xval - xlow) / (xhigh - xlow);
  return ylow + (yhigh - ylow) * (pw == 1.0 ? t : pow(t, pw));
}
__device__ __forceinline__ double gcum_d(double x) { return 0.5 * erfc(-x / 1.4142135623730951); }
__device__ __forceinline__ double backtr_value(const BackTr& B, double y) {
  const double* gt = B.gt;
  const double* vr = B.vr;
  const int nt = B.nt;
  if (y <= gt[0]) {
    const double cdflo = gcum_d(gt[0]), cdfbt = gcum_d(y);
    double z = powint_d(0.0, cdflo, B.zmin, vr[0], cdfbt, B.lt == 2 ? B.ltp : 1.0);
    if (nt == 1) z = vr[0];
    return z;
  }
  if (y >= gt[nt - 1]) {
    const double cdfhi = gcum_d(gt[nt - 1]), cdfbt = gcum_d(y);
    if (B.ut == 2) return powint_d(cdfhi, 1.0, vr[nt - 1], B.zmax, cdfbt, B.utp);
    if (B.ut == 4) {
      const double lam = pow(vr[nt - 1], B.utp) * (1.0 - cdfhi);
      return pow(lam / fmax(1.0 - cdfbt, 1.0e-300), 1.0 / B.utp);
    }
    return powint_d(cdfhi, 1.0, vr[nt - 1], B.zmax, cdfbt, 1.0);
  }
  int lo;
  if (B.base) {
    const double f = (y - B.g0) * B.inv_w;
    const int kb = f <= 0.0 ? 0 : (f >= (double)B.nbucket ? B.nbucket - 1 : (int)f);
    int c = B.base[kb];   // a generic load: the table may be in shared memory
    while (c > 0 && gt[c - 1] > y) --c;
    while (c < nt && gt[c] <= y) ++c;
    lo = c;
  } else {
    lo = 1;
    int hi = nt;
    while (hi - lo > 1) {
      const int mid = (lo + hi) / 2;
      if (gt[mid - 1] <= y) lo = mid;
      else hi = mid;
    }
  }
  return powint_d(gt[lo - 1], gt[lo], vr[lo - 1], vr[lo], y, 1.0);
}
__device__ __forceinline__ double backtr_apply(const BackTr& B, double y) {
  return B.mode == 1 ? backtr_value(B, y) : (B.mode == 2 ? y + B.skmean : y);
}

__global__ void k_backtr(double* __restrict__ res, long long tot, BackTr B) {
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x)
    res[q] = backtr_apply(B, res[q]);
}
// the same with the table (gt, vr and the bucket index) copied into the
// shared memory of each block of a resident grid: the lookups of one value
// are dependent loads, which shared memory serves with far less latency
__host__ __device__ inline size_t backtr_smem_bytes(int nt, int nbucket) {
  return (size_t)nt * 16 + (size_t)(nbucket + 1) * 4;
}
__global__ void __launch_bounds__(256) k_backtr_smem(double* __restrict__ res, long long tot, BackTr B) {
  extern __shared__ __align__(16) unsigned char smb[];
  double* sgt = reinterpret_cast<double*>(smb);
  double* svr = sgt + B.nt;
  int* sbase = reinterpret_cast<int*>(svr + B.nt);
  for (int q = threadIdx.x; q < B.nt; q += blockDim.x) {
    sgt[q] = B.gt[q];
    svr[q] = B.vr[q];
  }
  if (B.base)
    for (int q = threadIdx.x; q <= B.nbucket; q += blockDim.x) sbase[q] = B.base[q];
  __syncthreads();
  BackTr S = B;
  S.gt = sgt;
  S.vr = svr;
  S.base = B.base ? sbase : nullptr;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x)
    res[q] = backtr_apply(S, res[q]);
}

// ---------------------------------------------------------------- kriging, rows in registers
// The same kriging for ndmax <= 32, with the system of a node held by one warp
// in registers: lane r owns row r of the covariance matrix (NDT >= ndmax
// doubles, or floats in the FP32 form).  Column step c of the right-looking
// Cholesky: the pivot comes from lane c by a shuffle, each lane scales its
// element of column c by the pivot's reciprocal square root, the scaled
// column goes to a shared-memory vector (two alternating buffers, one warp
// barrier per column) and every lane updates its row with it from registers.
// The forward substitution L y = b runs in the same loop; the back
// substitution L^T w = y reads the transpose of L from shared memory.  Lanes
// and columns past the node's neighbour count hold values that no valid
// entry ever reads.  FP32 form: FP32 factor and solves, the FP64 matrix kept
// in shared memory for the residual of one refinement step.  Same ridge rule,
// neighbour order and counters as k_cond_krige.
template <int PREC, int NDT> struct KregLayout {
  using T = typename std::conditional<PREC == 0, double, float>::type;
  static constexpr int PITCH = NDT + 1;
  static constexpr int LAT = 0;                                            // int4 per neighbour
  static constexpr int W = LAT + 16 * NDT;                                 // double w
  static constexpr int COL = W + 8 * NDT;                                  // 2 x 32 T
  static constexpr int LS = COL + 2 * 32 * (int)sizeof(T);                 // NDT x PITCH T (transpose of L)
  static constexpr int AS = (LS + NDT * PITCH * (int)sizeof(T) + 15) & ~15; // NDT x PITCH double (FP32 form)
  static constexpr int BYTES = ((PREC == 0 ? AS : AS + NDT * PITCH * 8) + 15) & ~15;
};

// CTAs per SM asked of the register allocator for NDT = 32 (the smaller
// classes ask for 3)
#ifndef KREG_MINB32
#define KREG_MINB32 2
#endif
// the strict lower triangle of an NDT x NDT system: entries, and entries per lane
template <int NDT> struct KregTri {
  static constexpr int NE = NDT * (NDT - 1) / 2;
  static constexpr int NIT = (NE + 31) / 32;
};

template <int PREC, int NDT, int MINB>
__global__ void __launch_bounds__(256, MINB) k_cond_krige_reg(CondGeo G, const KModel* __restrict__ mdl, CovTab ctab,
                                                        long long node0,
                                                        int count, const int* __restrict__ nbr,
                                                        const int* __restrict__ nnb, const int* __restrict__ ixs,
                                                        const int* __restrict__ iys, const int* __restrict__ izs,
                                                        const double* __restrict__ dg,
                                                        const double* __restrict__ simd, double* __restrict__ res,
                                                        unsigned long long* __restrict__ counters) {
  using Ly = KregLayout<PREC, NDT>;
  using KT = KregTri<NDT>;
  using T = typename Ly::T;
  constexpr int PITCH = Ly::PITCH;
  constexpr int KV = 16 / (int)sizeof(T);   // column elements per 16-byte load
  static_assert(NDT % KV == 0 && Ly::COL % 16 == 0 && Ly::BYTES % 16 == 0, "16-byte column loads");
  extern __shared__ __align__(16) unsigned char smk[];
  __shared__ unsigned long long bcount[4];
  __shared__ unsigned short tri[KT::NE > 0 ? KT::NE : 1];   // (r << 8) | c of entry e
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int nwb = blockDim.x >> 5;
  if (threadIdx.x < 4) bcount[threadIdx.x] = 0;
  for (int r = 1 + (int)threadIdx.x; r < NDT; r += blockDim.x)
    for (int c = 0; c < r; ++c) tri[r * (r - 1) / 2 + c] = (unsigned short)((r << 8) | c);
  const double c00 = cov_lat_g(ctab, mdl, 0, 0, 0, G.dx, G.dy, G.dz);
  __syncthreads();
  unsigned char* mine = smk + (size_t)Ly::BYTES * wib;
  int4* lat = reinterpret_cast<int4*>(mine + Ly::LAT);
  double* wsm = reinterpret_cast<double*>(mine + Ly::W);
  T* colb = reinterpret_cast<T*>(mine + Ly::COL);
  T* Ls = reinterpret_cast<T*>(mine + Ly::LS);
  double* As = reinterpret_cast<double*>(mine + Ly::AS);   // FP32 form only
  const long long M = (long long)G.nx * G.ny * G.nz;
  for (int q = blockIdx.x * nwb + wib; q < count; q += gridDim.x * nwb) {
    const long long node = node0 + q;
    const int code = nnb[q];
    const int nn = code & 0xffff, exact = code >> 16;
    if (lane == 0) atomicAdd_block(&bcount[0], (unsigned long long)nn);
    if (nn == 0) {
      if (lane == 0) atomicAdd_block(&bcount[2], 1ull);
      continue;
    }
    const int* nl = nbr + (long long)q * G.ndmax;
    if (exact) {
      const double v = dg[nl[0]];
      for (int l = lane; l < G.nreal; l += 32) res[node + M * l] = v;
      if (lane == 0) atomicAdd_block(&bcount[3], 1ull);
      continue;
    }
    // a conditioned grid has at most 2^27 nodes: 32-bit index arithmetic
    const uint32_t nu = (uint32_t)node, row = nu / (uint32_t)G.nx;
    const int i = (int)(nu - row * (uint32_t)G.nx), j = (int)(row % (uint32_t)G.ny), k = (int)(row / (uint32_t)G.ny);
    const bool act = lane < nn;
    int4 me = make_int4(0, 0, 0, 0);
    if (act) {
      const int cp = nl[lane];
      me = make_int4(__ldg(ixs + cp) - 1, __ldg(iys + cp) - 1, __ldg(izs + cp) - 1, cp);
      lat[lane] = me;
    }
    __syncwarp();
    const double b = act ? cov_lat_g(ctab, mdl, me.x - i, me.y - j, me.z - k, G.dx, G.dy, G.dz) : 0.0;
    // A in shared memory (FP64 in As for the FP32 form, else in Ls): the
    // strict lower triangle spread over the lanes (entry e = r (r-1)/2 + c,
    // c < r < nn), every table load of a lane issued before any is used, the
    // lags outside the table evaluated afterwards, each value stored at (r, c)
    // and (c, r) (C(h) = C(-h) holds bitwise: the rotated components of -h are
    // the negated components of h); the diagonal is C(0).  Entries of rows or
    // columns past nn are not written: no valid entry reads them.
    {
      double* A = PREC == 1 ? As : reinterpret_cast<double*>(Ls);
      const int ne = nn * (nn - 1) / 2;
      double v[KT::NIT];
      int rc[KT::NIT];
      bool far[KT::NIT];
#pragma unroll
      for (int it = 0; it < KT::NIT; ++it) {
        const int e = lane + 32 * it;
        rc[it] = e < ne ? (int)tri[e] : 0;
        const int4 o = lat[rc[it] >> 8], p = lat[rc[it] & 255];
        int di = o.x - p.x, dj = o.y - p.y, dk = o.z - p.z;
        if (dk < 0) {
          di = -di;
          dj = -dj;
          dk = -dk;
        }
        far[it] = !(ctab.v && dk <= ctab.tz && abs(dj) <= ctab.ty && abs(di) <= ctab.tx);
        const size_t off =
            (size_t)(di + ctab.tx) + (size_t)(2 * ctab.tx + 1) * ((dj + ctab.ty) + (size_t)(2 * ctab.ty + 1) * dk);
        v[it] = far[it] ? 0.0 : __ldg(ctab.v + off);
      }
#pragma unroll
      for (int it = 0; it < KT::NIT; ++it) {
        const int e = lane + 32 * it;
        if (e < ne) {
          const int r = rc[it] >> 8, c = rc[it] & 255;
          if (far[it]) {   // outside the table (or no table): evaluated directly
            const int4 o = lat[r], p = lat[c];
            v[it] = cov_lat_g(ctab, mdl, o.x - p.x, o.y - p.y, o.z - p.z, G.dx, G.dy, G.dz);
          }
          if constexpr (PREC == 1) {
            A[r * PITCH + c] = v[it];
            A[c * PITCH + r] = v[it];
          } else {
            Ls[r * PITCH + c] = v[it];
            Ls[c * PITCH + r] = v[it];
          }
        }
      }
      if (act) {
        if constexpr (PREC == 1)
          A[lane * PITCH + lane] = c00;
        else
          Ls[lane * PITCH + lane] = c00;
      }
      // fewer neighbours than NDT: the system is padded to NDT with identity
      // rows and columns (and zero right-hand sides), so that every step below
      // runs for all NDT columns without a test.  A padded column's entries in
      // the real rows are exact zeros, so every update it makes subtracts an
      // exact zero: the real entries of L, y and w keep their bits.
      if (nn < NDT) {
        for (int e = lane; e < NDT * NDT; e += 32) {
          const int r = e / NDT, c = e - r * NDT;
          if (r >= nn || c >= nn) {
            if constexpr (PREC == 1)
              A[r * PITCH + c] = r == c ? 1.0 : 0.0;
            else
              Ls[r * PITCH + c] = r == c ? 1.0 : 0.0;
          }
        }
      }
    }
    __syncwarp();
    double ridge = 1.0e-10 * G.c0;
    T a[NDT];
    T myinv = T(0), yv = T(0);
    bool good = false;
    int tries;
    for (tries = 1; tries <= 3; ++tries) {
      // row `lane` of A + ridge I into registers (identity rows for lanes past nn)
#pragma unroll
      for (int c = 0; c < NDT; ++c) {
        double v = 0.0;
        if (lane < NDT) v = PREC == 1 ? As[lane * PITCH + c] : (double)Ls[lane * PITCH + c];
        if (c == lane) v = act ? v + ridge : 1.0;
        a[c] = (T)v;
      }
      T bcur = (T)b;
      good = true;
#pragma unroll
      for (int c = 0; c < NDT; ++c) {
        const T piv = __shfl_sync(0xffffffffu, a[c], c);
        // the same value in every lane; a failed factor is recomputed from
        // A (with a larger ridge), so the steps after a failure only waste work
        good = good && piv > T(0);
        const T inv = rsqrt_nr(piv);
        const T lrc = a[c] * inv;
        a[c] = lrc;
        if (lane == c) myinv = inv;
        T* cb = colb + (c & 1) * 32;
        cb[lane] = lrc;
        __syncwarp();
        const T yc = __shfl_sync(0xffffffffu, bcur * inv, c);
        if (lane == c) yv = yc;
        bcur = fma(-lrc, yc, bcur);
#pragma unroll
        for (int k0 = (c + 1) / KV * KV; k0 < NDT; k0 += KV) {
          // the column 16 bytes at a time (every lane reads the same words:
          // one wavefront per load); elements up to c are loaded, not used
          T cv[KV];
          *reinterpret_cast<uint4*>(cv) = *reinterpret_cast<const uint4*>(cb + k0);
#pragma unroll
          for (int u = 0; u < KV; ++u)
            if (k0 + u > c) a[k0 + u] = fma(-lrc, cv[u], a[k0 + u]);
        }
      }
      if (good) break;
      ridge = ridge * 1.0e3;
      __syncwarp();
    }
    if (!good) {
      if (lane == 0) atomicAdd_block(&bcount[1], 1ull);
      continue;
    }
    if (tries > 1 && lane == 0) atomicAdd_block(&bcount[1], 1ull);
    // back substitution L^T w = y with the transpose of L in shared memory
    if (lane < NDT) {
#pragma unroll
      for (int c = 0; c < NDT; ++c) Ls[lane * PITCH + c] = a[c];
    }
    __syncwarp();
    T acc = yv, w = T(0);
#pragma unroll
    for (int r = NDT - 1; r >= 0; --r) {
      const T wr = __shfl_sync(0xffffffffu, acc * myinv, r);
      if (lane == r) w = wr;
      if (lane < r) acc = fma(-Ls[r * PITCH + lane], wr, acc);
    }
    if (lane < NDT) wsm[lane] = (double)w;   // 0 in padded rows
    __syncwarp();
    if constexpr (PREC == 1) {
      // one refinement: residual b - (A + ridge I) w in FP64, then
      // L L^T d = residual in FP32 and w += d
      double rres = 0.0;
      if (act) {
        rres = b - ridge * wsm[lane];
        // the padded columns add exact zeros (A and w are 0 there)
#pragma unroll
        for (int c0 = 0; c0 < NDT; c0 += 2) {
          const double2 wv = *reinterpret_cast<const double2*>(wsm + c0);
          rres -= As[lane * PITCH + c0] * wv.x;
          rres -= As[lane * PITCH + c0 + 1] * wv.y;
        }
      }
      T dcur = (T)rres, dy = T(0);
#pragma unroll
      for (int c = 0; c < NDT; ++c) {
        const T yc = __shfl_sync(0xffffffffu, dcur * myinv, c);
        if (lane == c) dy = yc;
        dcur = fma(-a[c], yc, dcur);
      }
      T acc2 = dy, d = T(0);
#pragma unroll
      for (int r = NDT - 1; r >= 0; --r) {
        const T wr = __shfl_sync(0xffffffffu, acc2 * myinv, r);
        if (lane == r) d = wr;
        if (lane < r) acc2 = fma(-Ls[r * PITCH + lane], wr, acc2);
      }
      __syncwarp();
      if (act) wsm[lane] += (double)d;
      __syncwarp();
    }
    double zk = act ? wsm[lane] * dg[me.w] : 0.0;   // sum of w dg: a butterfly over the lanes
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) zk += __shfl_xor_sync(0xffffffffu, zk, off);
    for (int l = lane; l < G.nreal; l += 32) {
      // all gathers of the realization first, then the sum in neighbour order
      double sv[NDT];
#pragma unroll
      for (int p = 0; p < NDT; ++p) sv[p] = p < nn ? simd[(long long)lat[p].w * G.nreal + l] : 0.0;
      const double rv = res[node + M * l];
      double sks = 0.0;
#pragma unroll
      for (int p = 0; p < NDT; ++p)
        if (p < nn) sks += wsm[p] * sv[p];
      res[node + M * l] = zk + rv - sks;
    }
    __syncwarp();
  }
  __syncthreads();
  if (threadIdx.x < 4 && bcount[threadIdx.x]) atomicAdd(&counters[threadIdx.x], bcount[threadIdx.x]);
}

__global__ void k_gather_simd(const double* __restrict__ res, long long M, const int* __restrict__ ix,
                              const int* __restrict__ iy, const int* __restrict__ iz, int nd, int nreal, int nx, int ny,
                              double* __restrict__ simd) {
  // simd[d * nreal + l]: the realizations of one datum side by side, so that
  // the lanes of a kriging warp (one realization each) read whole lines
  const long long tot = (long long)nd * nreal;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot; q += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(q % nreal), d = (int)(q / nreal);
    simd[q] = res[(ix[d] - 1) + (long long)nx * ((iy[d] - 1) + (long long)ny * (iz[d] - 1)) + M * l];
  }
}

const void* module_anchor_cond() { return reinterpret_cast<const void*>(k_gather_simd); }

}  // namespace ss3d

using namespace ss3d;

// ---------------------------------------------------------------- host helpers
namespace {

int fnint(double x) { return (int)lround(x); }   // Fortran nint: half away from zero

// GSLIB-style heapsort of an index array by key (sift-down heap, ascending);
// the same algorithm as the reference so that ties end in the same order
void heapsort_idx(const double* key, int* idx, int n) {
  auto sift = [&](int root, int last) {
    int parent = root;
    int v = idx[parent - 1];
    for (;;) {
      int child = 2 * parent;
      if (child > last) break;
      if (child < last && key[idx[child] - 1] > key[idx[child - 1] - 1]) child = child + 1;
      if (key[idx[child - 1] - 1] > key[v - 1]) {
        idx[parent - 1] = idx[child - 1];
        parent = child;
      } else {
        break;
      }
    }
    idx[parent - 1] = v;
  };
  for (int i = n / 2; i >= 1; i--) sift(i, n);
  for (int i = n; i >= 2; i--) {
    std::swap(idx[0], idx[i - 1]);
    sift(1, i - 1);
  }
}

// idx (1-based) ordered by key, as heapsort_idx orders it whenever no key
// occurs more than max_tie times: distinct keys have one sorted order, so a
// comparison sort with any tie rule gives heapsort's permutation up to the
// order inside groups of equal keys, which a caller that tolerates max_tie
// equal keys does not see (the merge of data on one node sums a group, and a
// sum of two is the same in either order).  Larger groups take the heapsort
// itself, so the result is always one a caller cannot tell from it.
void sort_idx(const double* key, int* idx, int n, int max_tie) {
  // LSD radix sort, 8 bits a pass, on the doubles' bits mapped to an order-
  // preserving unsigned key (sign bit set for positives, all bits flipped for
  // negatives; -0 is taken as +0, which the comparisons of heapsort equal)
  std::vector<uint64_t> k(n), k2(n);
  std::vector<int> v(n), v2(n);
  for (int q = 0; q < n; q++) {
    uint64_t b;
    std::memcpy(&b, &key[idx[q] - 1], 8);
    if (b == 0x8000000000000000ull) b = 0;
    k[q] = (b >> 63) ? ~b : (b | 0x8000000000000000ull);
    v[q] = idx[q];
  }
  uint64_t diff = 0;   // bits that differ between keys: passes over constant bytes are skipped
  for (int q = 1; q < n; q++) diff |= k[q] ^ k[0];
  for (int sh = 0; sh < 64; sh += 8) {
    if (!((diff >> sh) & 0xff)) continue;
    int cnt[257] = {0};
    for (int q = 0; q < n; q++) cnt[((k[q] >> sh) & 0xff) + 1]++;
    for (int c = 0; c < 256; c++) cnt[c + 1] += cnt[c];
    for (int q = 0; q < n; q++) {
      const int d = cnt[(k[q] >> sh) & 0xff]++;
      k2[d] = k[q];
      v2[d] = v[q];
    }
    k.swap(k2);
    v.swap(v2);
  }
  int run = 1;
  for (int q = 1; q < n; q++) {
    run = k[q] == k[q - 1] ? run + 1 : 1;
    if (run > max_tie) {
      heapsort_idx(key, idx, n);
      return;
    }
  }
  for (int q = 0; q < n; q++) idx[q] = v[q];
}

// inverse standard normal cdf: Acklam's rational approximation refined by one
// Halley step on erfc (as the reference's gauinv)
double gauinv(double p0) {
  static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                              1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
  static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                              6.680131188771972e+01, -1.328068155288572e+01};
  static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                              -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
  static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                              3.754408661907416e+00};
  const double p = std::min(std::max(p0, 1.0e-15), 1.0 - 1.0e-15);
  double x;
  if (p < 0.02425) {
    const double q = sqrt(-2.0 * log(p));
    x = (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
        ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0);
  } else if (p <= 1.0 - 0.02425) {
    const double q = p - 0.5, r = q * q;
    x = (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
        (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1.0);
  } else {
    const double q = sqrt(-2.0 * log(1.0 - p));
    x = -((((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
          ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1.0));
  }
  const double e = 0.5 * erfc(-x / 1.4142135623730951) - p;
  const double u = e * 2.5066282746310002 * exp(0.5 * x * x);
  return x - u / (1.0 + 0.5 * x * u);
}

// Temporaries of one call from the stream-ordered pool of the call's stream:
// freeing them does not synchronise the device, so other threads' streams
// keep running.
struct DevBuf {
  cudaStream_t st;
  std::vector<void*> ptrs;
  explicit DevBuf(cudaStream_t s) : st(s) {}
  ~DevBuf() {
    for (void* p : ptrs) cudaFreeAsync(p, st);
  }
  template <typename T>
  cudaError_t alloc(T** p, size_t n) {
    cudaError_t e = cudaMallocAsync((void**)p, sizeof(T) * std::max<size_t>(n, 1), st);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

}  // namespace

namespace {
// Staging buffer of the conditioning calls of this host thread, in pageable
// memory.  A page-locked allocation would serialise the work of every stream
// of the device (an implicit synchronisation of cudaMallocHost), which in a
// serving loop stalls the requests of the other slots behind a running
// kriging call; a copy from pageable memory is staged by the driver without
// such a synchronisation.
thread_local std::vector<unsigned char> g_cond_stage;

cudaError_t cond_stage(size_t bytes, unsigned char** out) {
  if (g_cond_stage.size() < bytes) g_cond_stage.resize(std::max(bytes, (size_t)1 << 20));
  *out = g_cond_stage.data();
  return cudaSuccess;
}

// min of v^T Q v over the box lo <= v <= hi (Q symmetric positive definite),
// exactly, by its active sets: each coordinate at its lower bound, at its
// upper bound or free, the free ones solving the reduced stationarity
// equations; -inf when a reduced system is singular (no pruning then).  Stops
// at the first value <= stop (the caller only asks whether the min is).
double box_min_quad(const double Q[3][3], const double lo[3], const double hi[3], double stop) {
  double best = INFINITY;
  for (int code = 0; code < 27; ++code) {
    const int st[3] = {code % 3, (code / 3) % 3, code / 9};   // 0 lower, 1 upper, 2 free
    double v[3];
    int fr[3], nf = 0;
    for (int a = 0; a < 3; ++a) {
      v[a] = st[a] == 0 ? lo[a] : (st[a] == 1 ? hi[a] : 0.0);
      if (st[a] == 2) fr[nf++] = a;
    }
    if (nf > 0) {
      double A[3][4];
      for (int i = 0; i < nf; ++i) {
        double b = 0.0;
        for (int a = 0; a < 3; ++a)
          if (st[a] != 2) b -= Q[fr[i]][a] * v[a];
        for (int j = 0; j < nf; ++j) A[i][j] = Q[fr[i]][fr[j]];
        A[i][nf] = b;
      }
      for (int c = 0; c < nf; ++c) {   // Gaussian elimination, partial pivoting
        int pr = c;
        for (int r = c + 1; r < nf; ++r)
          if (fabs(A[r][c]) > fabs(A[pr][c])) pr = r;
        if (!(fabs(A[pr][c]) > 1e-300)) return -INFINITY;
        for (int j = 0; j <= nf; ++j) std::swap(A[c][j], A[pr][j]);
        for (int r = 0; r < nf; ++r)
          if (r != c) {
            const double f = A[r][c] / A[c][c];
            for (int j = c; j <= nf; ++j) A[r][j] -= f * A[c][j];
          }
      }
      bool inside = true;
      for (int i = 0; i < nf; ++i) {
        v[fr[i]] = A[i][nf] / A[i][i];
        if (v[fr[i]] < lo[fr[i]] || v[fr[i]] > hi[fr[i]]) inside = false;
      }
      if (!inside) continue;
    }
    double q = 0.0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) q += v[a] * Q[a][b] * v[b];
    best = std::min(best, q);
    if (best <= stop) break;
  }
  return best;
}

// The super-block offsets of the search box by rows along x, in the
// reference's scan order (z, then y offset ascending), each row the x offsets
// from its first to its last block that may hold a point inside the search
// ellipsoid for some node of the centre block (rows with none are dropped).
// A node and a datum whose blocks differ by o along an axis differ by a lag
// in ((o - 1) bs, (o + 1) bs) along it (both are assigned to blocks by the
// same shifted floor); the box is widened by 1e-6 bs for the rounding of that
// assignment, and a block may hold such a point unless the smallest |R v|^2
// over the box exceeds rmax^2 by more than 1e-9 relative (R the search
// rotation, the d2 of the candidates being |R h|^2 / rmax^2).  Blocks between
// the first and last of a row are scanned whatever their test: a block
// scanned needlessly only adds rejected candidates.  Search boxes of more than
// 4096 blocks keep every block.
void super_block_rows(const CondGeo& G, std::vector<int4>& rows) {
  const long long tot = (2LL * G.mbx + 1) * (2LL * G.mby + 1) * (2LL * G.mbz + 1);
  double Q[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      double v = 0.0;
      for (int k = 0; k < 3; ++k) v += G.rot[3 * k + r] * G.rot[3 * k + c];
      Q[r][c] = v;
    }
  const double bs[3] = {G.bsx, G.bsy, G.bsz};
  for (int dk = -G.mbz; dk <= G.mbz; ++dk)
    for (int dj = -G.mby; dj <= G.mby; ++dj) {
      int lo_i = G.mbx + 1, hi_i = -G.mbx - 1;
      for (int di = -G.mbx; di <= G.mbx; ++di) {
        bool keep = tot > 4096;
        if (!keep) {
          const int o[3] = {di, dj, dk};
          double lo[3], hi[3];
          for (int a = 0; a < 3; ++a) {
            lo[a] = (o[a] - 1) * bs[a] - 1e-6 * bs[a];
            hi[a] = (o[a] + 1) * bs[a] + 1e-6 * bs[a];
          }
          const double lim = G.rmax2 * (1.0 + 1e-9);
          keep = box_min_quad(Q, lo, hi, lim) <= lim;
        }
        if (keep) {
          lo_i = std::min(lo_i, di);
          hi_i = std::max(hi_i, di);
        }
      }
      if (lo_i <= hi_i) rows.push_back(make_int4(lo_i, hi_i, dj, dk));
    }
}
}  // namespace

extern "C" int ss3d_condition(double* res, const int n[3], int nreal, const double xmin3[3], const double d3[3],
                              const ss3d_struct* st, int nst, double nugget, const ss3d_cond_params* cp,
                              const double* rows, int nrows, int nvar, int precision, ss3d_cond_stats* cs,
                              double* vrt_out, double* gtt_out, double* dxs_out, double* dys_out, double* dzs_out,
                              double* dval_out, double* dg_out) {
  if (!res || !n || !xmin3 || !d3 || !st || !cp || (!rows && nrows > 0))
    return set_error(SS3D_EINVAL, "NULL argument");
  if (nst < 1 || nst > MAXST) return set_error(SS3D_EINVAL, "nstruct out of range");
  if (cp->ndmax < 1 || cp->ndmax > 100) return set_error(SS3D_EINVAL, "cond: ndmax must be in 1..100");
  if (cp->radius[0] <= 0 || cp->radius[1] <= 0 || cp->radius[2] <= 0)
    return set_error(SS3D_EINVAL, "cond: search radii must be positive");
  if (precision != SS3D_FP64 && precision != SS3D_FP32) return set_error(SS3D_EINVAL, "unknown precision");
  auto colok = [&](int c, bool opt) { return (opt && c == 0) || (c >= 1 && c <= nvar); };
  if (!colok(cp->ixc, false) || !colok(cp->iyc, false) || !colok(cp->ivc, false) || !colok(cp->izc, true) ||
      !colok(cp->iwc, true))
    return set_error(SS3D_EINVAL, "cond: data column out of range");
  const int nx = n[0], ny = n[1], nz = n[2];
  const double xmin = xmin3[0], ymin = xmin3[1], zmin = xmin3[2];
  const double dx = d3[0], dy = d3[1], dz = d3[2];
  // search ellipsoid as a unit-sill spherical structure (f90:754-758)
  ss3d_struct srch{1, 1.0, cp->radius[0], cp->radius[1], cp->radius[2], cp->angles[0], cp->angles[1], cp->angles[2]};
  double srot[3][3], saxes[3][3];
  setrot_public(srch, srot, saxes);
  const double ex = sqrt(saxes[0][0] * saxes[0][0] + saxes[1][0] * saxes[1][0] + saxes[2][0] * saxes[2][0]);
  const double ey = sqrt(saxes[0][1] * saxes[0][1] + saxes[1][1] * saxes[1][1] + saxes[2][1] * saxes[2][1]);
  const double ez = sqrt(saxes[0][2] * saxes[0][2] + saxes[1][2] * saxes[1][2] + saxes[2][2] * saxes[2][2]);
  // ---- snap to nodes, trim, drop data outside the grid (f90:782-804)
  std::vector<double> raw;
  std::vector<double> key;
  raw.reserve((size_t)nrows * 5);
  key.reserve((size_t)nrows);
  int nn = 0, nout = 0;
  for (int q = 0; q < nrows; q++) {
    const double* row = rows + (size_t)q * nvar;
    const double v = row[cp->ivc - 1];
    if (v < cp->tmin || v >= cp->tmax) continue;
    const int j = fnint((row[cp->ixc - 1] - xmin) / dx) + 1;
    const int k = fnint((row[cp->iyc - 1] - ymin) / dy) + 1;
    int r = 1;
    if (cp->izc > 0 && nz > 1) r = fnint((row[cp->izc - 1] - zmin) / dz) + 1;
    if (j < 1 || j > nx || k < 1 || k > ny || r < 1 || r > nz) {
      nout++;
      continue;
    }
    raw.push_back(j);
    raw.push_back(k);
    raw.push_back(r);
    raw.push_back(v);
    raw.push_back(cp->iwc > 0 ? row[cp->iwc - 1] : 1.0);
    key.push_back((double)j + (double)nx * ((double)(k - 1) + (double)ny * (double)(r - 1)));
    nn++;
  }
  if (nn == 0) return set_error(SS3D_ENODATA, "cond: no conditioning data inside the grid");
  // ---- merge data of the same node (f90:805-828)
  std::vector<int> ord(nn);
  for (int q = 0; q < nn; q++) ord[q] = q + 1;
  sort_idx(key.data(), ord.data(), nn, 2);
  std::vector<int> ix, iy, iz;
  std::vector<double> dval, dwt;
  for (auto* vi : {&ix, &iy, &iz}) vi->reserve(nn);
  for (auto* vd : {&dval, &dwt}) vd->reserve(nn);
  for (int i = 1; i <= nn;) {
    int j = i;
    while (j < nn && key[ord[j] - 1] == key[ord[i - 1] - 1]) j++;
    const double* r0 = &raw[5 * (size_t)(ord[i - 1] - 1)];
    ix.push_back(fnint(r0[0]));
    iy.push_back(fnint(r0[1]));
    iz.push_back(fnint(r0[2]));
    double sw = 0.0, svw = 0.0;
    for (int q = i; q <= j; q++) sw = sw + raw[5 * (size_t)(ord[q - 1] - 1) + 4];
    for (int q = i; q <= j; q++) svw = svw + raw[5 * (size_t)(ord[q - 1] - 1) + 3] * raw[5 * (size_t)(ord[q - 1] - 1) + 4];
    dwt.push_back(sw);
    dval.push_back(svw / sw);
    i = j + 1;
  }
  const int nd = (int)ix.size();
  std::vector<double> dxs(nd), dys(nd), dzs(nd), dg(nd), vrt(nd), gtt(nd);
  for (int q = 0; q < nd; q++) {
    dxs[q] = xmin + (double)(ix[q] - 1) * dx;
    dys[q] = ymin + (double)(iy[q] - 1) * dy;
    dzs[q] = zmin + (double)(iz[q] - 1) * dz;
  }
  // ---- normal scores (f90:830-847, nscore f90:639-658)
  double dmean = 0.0, dvar = 0.0;
  int nt = nd;
  if (cp->itrans == 1) {
    std::vector<int> idx(nd);
    for (int q = 0; q < nd; q++) idx[q] = q + 1;
    sort_idx(dval.data(), idx.data(), nd, 1);
    double sw = 0.0;
    for (int q = 0; q < nd; q++) sw = sw + dwt[q];
    double cpv = 0.0, oldcp = 0.0;
    for (int q = 0; q < nd; q++) {
      cpv = cpv + dwt[idx[q] - 1] / sw;
      gtt[q] = gauinv(0.5 * (cpv + oldcp));
      vrt[q] = dval[idx[q] - 1];
      dg[idx[q] - 1] = gtt[q];
      oldcp = cpv;
    }
    double s = 0.0;
    for (int q = 0; q < nd; q++) s = s + dg[q];
    dmean = s / nd;
    double v = 0.0;
    for (int q = 0; q < nd; q++) v = v + (dg[q] - s / nd) * (dg[q] - s / nd);
    dvar = v / nd;
  } else {
    for (int q = 0; q < nd; q++) dg[q] = dval[q] - cp->skmean;
  }
  // ---- super blocks (f90:866-892)
  int nsbx = std::max(1, std::min(100, (int)ceil((double)nx * dx / (0.5 * ex))));
  int nsby = std::max(1, std::min(100, (int)ceil((double)ny * dy / (0.5 * ey))));
  int nsbz = std::max(1, std::min(100, (int)ceil((double)nz * dz / (0.5 * ez))));
  if (nz == 1) nsbz = 1;
  while ((double)nsbx * nsby * nsbz > 2.0e6) {
    nsbx = std::max(1, nsbx * 3 / 4);
    nsby = std::max(1, nsby * 3 / 4);
    nsbz = std::max(1, nsbz * 3 / 4);
  }
  const int nsb = nsbx * nsby * nsbz;
  const double bsx = (double)nx * dx / (double)nsbx, bsy = (double)ny * dy / (double)nsby,
               bsz = (double)nz * dz / (double)nsbz;
  const int mbx = (int)ceil(ex / bsx), mby = (int)ceil(ey / bsy), mbz = (int)ceil(ez / bsz);
  std::vector<int> sbstart(nsb + 1), sbcount(nsb, 0), sbidx(nd), sbof(nd);
  for (int q = 0; q < nd; q++) {
    const int b1 = std::min(nsbx, std::max(1, (int)((dxs[q] - xmin + 0.5 * dx) / bsx) + 1));
    const int b2 = std::min(nsby, std::max(1, (int)((dys[q] - ymin + 0.5 * dy) / bsy) + 1));
    const int b3 = std::min(nsbz, std::max(1, (int)((dzs[q] - zmin + 0.5 * dz) / bsz) + 1));
    sbof[q] = b1 + nsbx * (b2 - 1 + nsby * (b3 - 1));
    sbcount[sbof[q] - 1]++;
  }
  sbstart[0] = 1;
  for (int q = 1; q <= nsb; q++) sbstart[q] = sbstart[q - 1] + sbcount[q - 1];
  std::fill(sbcount.begin(), sbcount.end(), 0);
  for (int q = 0; q < nd; q++) {
    const int b = sbof[q];
    sbidx[sbstart[b - 1] + sbcount[b - 1] - 1] = q + 1;
    sbcount[b - 1]++;
  }
  Model mdl;
  model_public(st, nst, nugget, mdl);
  KModel kmdl{};
  kmdl.nst = mdl.nst;
  kmdl.nugget = mdl.nugget;
  for (int q = 0; q < mdl.nst; q++) {
    kmdl.itype[q] = mdl.itype[q];
    kmdl.sill[q] = mdl.sill[q];
    for (int e = 0; e < 9; e++) kmdl.rots[q][e] = mdl.rot[q][e] / mdl.ahmax[q];
  }
  CondGeo G{};
  G.nx = nx;
  G.ny = ny;
  G.nz = nz;
  G.nreal = nreal;
  G.nd = nd;
  G.ndmax = cp->ndmax;
  G.xmin = xmin;
  G.ymin = ymin;
  G.zmin = zmin;
  G.dx = dx;
  G.dy = dy;
  G.dz = dz;
  G.nsbx = nsbx;
  G.nsby = nsby;
  G.nsbz = nsbz;
  G.mbx = mbx;
  G.mby = mby;
  G.mbz = mbz;
  G.bsx = bsx;
  G.bsy = bsy;
  G.bsz = bsz;
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) G.rot[3 * r + c] = srot[r][c];
  G.rmax2 = cp->radius[0] * cp->radius[0];
  G.c0 = covariance(mdl, 0.0, 0.0, 0.0);
  std::vector<int4> srows;
  super_block_rows(G, srows);
  G.nrow = (int)srows.size();
  // ---- device work
  cudaStream_t stm = current_stream();
  const long long M = (long long)nx * ny * nz;
  int cur_dev = 0;
  if (cudaGetDevice(&cur_dev) != cudaSuccess) return set_error(SS3D_ECUDA, "no current CUDA device");
  bool dev_res = false;
  if (int rc = check_ptr(res, cur_dev, sizeof(double), "res", &dev_res)) return rc;
  DevBuf bufs(stm);
  double* dres = res;
  cudaError_t e = cudaSuccess;
  if (!dev_res) {
    e = bufs.alloc(&dres, (size_t)M * nreal);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dres, res, sizeof(double) * M * nreal, cudaMemcpyHostToDevice, stm);
  }
  // The arrays of the call live in one device allocation; the ones that come
  // from the host go up in one copy, packed into a staging buffer of this
  // thread (kept between calls: a call ends with its stream synchronized, so
  // the buffer is free when the next one starts), which also takes the
  // counters back.
  const int chunk = (int)std::min<long long>(M, std::max<long long>(1, ((long long)1 << 30) / (4LL * cp->ndmax + 4)));
  size_t top = 0;
  auto place = [&](size_t bytes) {
    const size_t o = top;
    top = (top + bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t o_dg = place(sizeof(double) * nd), o_ix = place(sizeof(int) * nd), o_iy = place(sizeof(int) * nd),
               o_iz = place(sizeof(int) * nd), o_sbs = place(sizeof(int) * (nsb + 1)),
               o_sxyz = place(sizeof(double4) * nd), o_rows = place(sizeof(int4) * srows.size()),
               o_vr = place(sizeof(double) * nd), o_gt = place(sizeof(double) * nd), o_mdl = place(sizeof(KModel)),
               o_cnt = place(sizeof(unsigned long long) * 4);
  // bucket index of the normal-score table for the back transform: one
  // bucket per entry over [gt[0], gt[nt-1]]
  const int nbucket = (cp->itrans == 1 && nt >= 2 && gtt[nt - 1] > gtt[0]) ? nt : 0;
  const size_t o_base = place(sizeof(int) * (size_t)(nbucket + 1));
  const size_t up_bytes = top;
  const size_t o_simd = place(sizeof(double) * nd * (size_t)nreal), o_nbr = place(sizeof(int) * (size_t)chunk * cp->ndmax),
               o_nnb = place(sizeof(int) * (size_t)chunk);
  unsigned char* stage = nullptr;
  if (e == cudaSuccess) e = cond_stage(up_bytes, &stage);
  if (e == cudaSuccess) {
    auto put = [&](size_t o, const void* src, size_t bytes) {
      if (bytes) memcpy(stage + o, src, bytes);
    };
    put(o_dg, dg.data(), sizeof(double) * nd);
    put(o_ix, ix.data(), sizeof(int) * nd);
    put(o_iy, iy.data(), sizeof(int) * nd);
    put(o_iz, iz.data(), sizeof(int) * nd);
    put(o_sbs, sbstart.data(), sizeof(int) * (nsb + 1));
    double4* sx = reinterpret_cast<double4*>(stage + o_sxyz);   // the data in super-block order, (x, y, z, id)
    for (int p = 0; p < nd; p++) {
      const int d = sbidx[p] - 1;
      sx[p] = make_double4(dxs[d], dys[d], dzs[d], (double)d);
    }
    put(o_rows, srows.data(), sizeof(int4) * srows.size());
    put(o_vr, vrt.data(), sizeof(double) * nd);
    put(o_gt, gtt.data(), sizeof(double) * nd);
    put(o_mdl, &kmdl, sizeof(KModel));
    memset(stage + o_cnt, 0, sizeof(unsigned long long) * 4);
    if (nbucket) {
      int* base = reinterpret_cast<int*>(stage + o_base);
      const double w = (gtt[nt - 1] - gtt[0]) / nbucket;
      for (int kb = 0; kb <= nbucket; kb++)
        base[kb] = (int)(std::upper_bound(gtt.begin(), gtt.begin() + nt, gtt[0] + kb * w) - gtt.begin());
    }
  }
  unsigned char* arena = nullptr;
  if (e == cudaSuccess) e = bufs.alloc(&arena, top);
  if (e == cudaSuccess) e = cudaMemcpyAsync(arena, stage, up_bytes, cudaMemcpyHostToDevice, stm);
  double* ddg = reinterpret_cast<double*>(arena + o_dg);
  int* dix = reinterpret_cast<int*>(arena + o_ix);
  int* diy = reinterpret_cast<int*>(arena + o_iy);
  int* diz = reinterpret_cast<int*>(arena + o_iz);
  int* dsbs = reinterpret_cast<int*>(arena + o_sbs);
  double4* dsxyz = reinterpret_cast<double4*>(arena + o_sxyz);
  int4* dsrow = reinterpret_cast<int4*>(arena + o_rows);
  double* dvr = reinterpret_cast<double*>(arena + o_vr);
  double* dgt = reinterpret_cast<double*>(arena + o_gt);
  KModel* dmdl = reinterpret_cast<KModel*>(arena + o_mdl);   // the register kernels read the model from global memory
  unsigned long long* dcnt = reinterpret_cast<unsigned long long*>(arena + o_cnt);
  double* dsimd = reinterpret_cast<double*>(arena + o_simd);
  int* dnbr = reinterpret_cast<int*>(arena + o_nbr);
  int* dnnb = reinterpret_cast<int*>(arena + o_nnb);
  BackTr bt{};
  bt.mode = cp->itrans == 1 ? 1 : (cp->skmean != 0.0 ? 2 : 0);
  bt.vr = dvr;
  bt.gt = dgt;
  bt.base = nbucket ? reinterpret_cast<const int*>(arena + o_base) : nullptr;
  bt.nt = nt;
  bt.nbucket = nbucket;
  bt.lt = cp->ltail;
  bt.ut = cp->utail;
  bt.zmin = cp->zmin;
  bt.zmax = cp->zmax;
  bt.ltp = cp->ltpar;
  bt.utp = cp->utpar;
  bt.skmean = cp->skmean;
  bt.g0 = nbucket ? gtt[0] : 0.0;
  bt.inv_w = nbucket ? nbucket / (gtt[nt - 1] - gtt[0]) : 0.0;
  if (e == cudaSuccess) {
    k_gather_simd<<<std::max(1, std::min(1024, (int)(((long long)nd * nreal + 255) / 256))), 256, 0, stm>>>(
        dres, M, dix, diy, diz, nd, nreal, nx, ny, dsimd);
    ++g_launch_count;
    e = cudaGetLastError();
  }
  // lattice covariance table over the lags two search half-extents wide
  // (at most the grid), when it stays below 128 MB
  CovTab ctab{nullptr, 0, 0, 0};
  double* dctab = nullptr;
  {
    auto half = [](double ext, double step, int n) {
      return (int)std::min<double>(n - 1, ceil(2.0 * ext / step) + 1.0);
    };
    const int tx = half(ex, dx, nx), ty = half(ey, dy, ny), tz = half(ez, dz, nz);
    const double cnt = (2.0 * tx + 1.0) * (2.0 * ty + 1.0) * (tz + 1.0);
    if (cnt * sizeof(double) <= (double)(128u << 20) && e == cudaSuccess) {
      const long long ncnt = (long long)cnt;
      e = bufs.alloc(&dctab, (size_t)ncnt);
      if (e == cudaSuccess) {
        k_cov_table<<<(int)std::min<long long>(148 * 16, (ncnt + 255) / 256), 256, 0, stm>>>(kmdl, dx, dy, dz, tx,
                                                                                           ty, tz, dctab);
        ++g_launch_count;
        e = cudaGetLastError();
      }
      ctab = CovTab{dctab, tx, ty, tz};
    }
  }
  // kriging kernel: rows in registers for ndmax <= 32 (compile-time classes
  // of 8, 16, 24, 32), else the shared-memory warp Cholesky; CTAs of at most
  // 8 warps, limited by the shared memory of one warp
  const bool fp32 = precision == SS3D_FP32;
  const int ndt = cp->ndmax <= 8 ? 8 : cp->ndmax <= 16 ? 16 : cp->ndmax <= 24 ? 24 : cp->ndmax <= 32 ? 32 : 0;
  const void* kfn = nullptr;
  size_t per = 0, kfix = 0;
  switch (ndt * 2 + (fp32 ? 1 : 0)) {
    case 16: kfn = (const void*)k_cond_krige_reg<0, 8, 3>; per = KregLayout<0, 8>::BYTES; break;
    case 17: kfn = (const void*)k_cond_krige_reg<1, 8, 3>; per = KregLayout<1, 8>::BYTES; break;
    case 32: kfn = (const void*)k_cond_krige_reg<0, 16, 3>; per = KregLayout<0, 16>::BYTES; break;
    case 33: kfn = (const void*)k_cond_krige_reg<1, 16, 3>; per = KregLayout<1, 16>::BYTES; break;
    case 48: kfn = (const void*)k_cond_krige_reg<0, 24, 3>; per = KregLayout<0, 24>::BYTES; break;
    case 49: kfn = (const void*)k_cond_krige_reg<1, 24, 3>; per = KregLayout<1, 24>::BYTES; break;
    case 64: kfn = (const void*)k_cond_krige_reg<0, 32, KREG_MINB32>; per = KregLayout<0, 32>::BYTES; break;
    case 65: kfn = (const void*)k_cond_krige_reg<1, 32, KREG_MINB32>; per = KregLayout<1, 32>::BYTES; break;
    default:
      kfn = fp32 ? (const void*)k_cond_krige<1> : (const void*)k_cond_krige<0>;
      per = cond_warp_bytes(cp->ndmax, fp32 ? 1 : 0);
      kfix = cond_tri_bytes(cp->ndmax);
  }
  const int wpb = (int)std::max<size_t>(1, std::min<size_t>(8, (size_t)(96 * 1024) / per));
  if (e == cudaSuccess) e = func_smem(kfn, kfix + per * wpb);
  for (long long node0 = 0; node0 < M && e == cudaSuccess; node0 += chunk) {
    const int count = (int)std::min<long long>(chunk, M - node0);
    auto search = [&](auto cap) {
      constexpr int CAP = decltype(cap)::value, BS = SearchCfg<CAP>::BS;
      k_cond_search<CAP><<<(unsigned)((count + BS - 1) / BS), BS, 0, stm>>>(G, node0, count, dsxyz, dsbs, dsrow, dix,
                                                                          diy, diz, dnbr, dnnb);
    };
    if (cp->ndmax <= 8)
      search(std::integral_constant<int, 8>());
    else if (cp->ndmax <= 16)
      search(std::integral_constant<int, 16>());
    else if (cp->ndmax <= 24)
      search(std::integral_constant<int, 24>());
    else if (cp->ndmax <= 32)
      search(std::integral_constant<int, 32>());
    else if (cp->ndmax <= 64)
      search(std::integral_constant<int, 64>());
    else
      search(std::integral_constant<int, 100>());
    ++g_launch_count;
    e = cudaGetLastError();
    if (e != cudaSuccess) break;
    // short blocks (wpb warps of one node each, four nodes per warp in turn in
    // the register kernels, whose block setup would otherwise be paid per
    // node): work of other streams, e.g. of a serving loop's higher-priority
    // requests, gets SMs as blocks finish
    const long long per_blk = (long long)wpb * (ndt ? 4 : 1);
    const int nblk = (int)(((long long)count + per_blk - 1) / per_blk);
    const size_t ksm = kfix + per * wpb;
    void* kargs_reg[] = {&G, &dmdl, &ctab, &node0, (void*)&count, &dnbr, &dnnb, &dix, &diy, &diz, &ddg, &dsimd,
                         &dres, &dcnt};
    void* kargs_old[] = {&G, &kmdl, &ctab, &node0, (void*)&count, &dnbr, &dnnb, &dix, &diy, &diz, &ddg, &dsimd,
                         &dres, &dcnt};
    void** kargs = ndt ? kargs_reg : kargs_old;
    e = cudaLaunchKernel(kfn, dim3((unsigned)nblk), dim3(32 * wpb), kargs, ksm, stm);
    ++g_launch_count;
    if (e == cudaSuccess) e = cudaGetLastError();
  }
  const long long tot = M * nreal;
  if (e == cudaSuccess && bt.mode) {
    const size_t tb = backtr_smem_bytes(nt, nbucket);
    if (bt.mode == 1 && tb <= (64u << 10)) {   // 4 blocks of 256 threads per SM
      // the attribute is set once, to the largest table: changing it while
      // instances run on other streams (a server's other slots) may wait for them
      e = func_smem((const void*)k_backtr_smem, 64u << 10);
      if (e == cudaSuccess) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cur_dev);
        k_backtr_smem<<<(int)std::min<long long>(4LL * nsm, (tot + 255) / 256), 256, tb, stm>>>(dres, tot, bt);
        ++g_launch_count;
        e = cudaGetLastError();
      }
    } else {
      k_backtr<<<(int)std::min<long long>(148 * 32, (tot + 255) / 256), 256, 0, stm>>>(dres, tot, bt);
      ++g_launch_count;
      e = cudaGetLastError();
    }
  }
  unsigned long long cnt[4] = {0, 0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(stage + o_cnt, dcnt, sizeof cnt, cudaMemcpyDeviceToHost, stm);
  if (e == cudaSuccess && !dev_res)
    e = cudaMemcpyAsync(res, dres, sizeof(double) * M * nreal, cudaMemcpyDeviceToHost, stm);
  // synchronized on every path: the staging buffer is free again on return
  const cudaError_t es = cudaStreamSynchronize(stm);
  if (e == cudaSuccess) e = es;
  if (e != cudaSuccess) {
    cudaGetLastError();
    return set_error(SS3D_ECUDA, (std::string("condition: ") + cudaGetErrorString(e)).c_str());
  }
  memcpy(cnt, stage + o_cnt, sizeof cnt);
  if (cs) {
    cs->nd = nd;
    cs->nmerged = nn - nd;
    cs->nout = nout;
    cs->nsb[0] = nsbx;
    cs->nsb[1] = nsby;
    cs->nsb[2] = nsbz;
    cs->nsum = (int64_t)cnt[0];
    cs->nfail = (int)cnt[1];
    cs->nnone = (int)cnt[2];
    cs->nexact = (int)cnt[3];
    cs->data_mean = dmean;
    cs->data_var = dvar;
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
  return SS3D_OK;
}
