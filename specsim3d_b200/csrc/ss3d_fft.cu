// ss3d_fft.cu -- spectrum construction and realization synthesis kernels.
//
// GPU replacement of these reference stages (src/specsim3d.f90):
//   covariance grid        f90:1256-1270  -> k_spec_rows   (fused with the x R2C pass)
//   forward fft3d, /ntot   f90:1273-1274  -> k_spec_rows, k_axis_c2c (y, z)
//   amp = sqrt(max(S,0))   f90:1275-1292  -> k_spec_amp (+ k_reduce_spec)
//   Hermitian fill         f90:1305-1334  -> k_axis_gen (fused into the first
//                                            inverse pass) or k_gen
//   inverse fft3d + crop   f90:1335-1340  -> k_axis_c2c (z, y), k_rows_c2r (x)
//
// Data layout in HBM: every complex grid is the Hermitian half spectrum
// i in [0, H), H = npx/2+1, stored as [k][j][HP] with row pitch HP = H rounded
// up to an even count (16-byte aligned rows of float2).  A batch of realizations
// stores its grids back to back, wstride elements apart.
//
// Each FFT kernel keeps one tile in shared memory: TX lines of the transformed
// axis (TX consecutive elements in memory, so that every global access of a
// warp covers whole 32-byte sectors) and runs the radix-8/4/2 Stockham engine
// of ss3d_device.cuh on it.  Only the positions that survive the final crop are
// written back (z pass: k < nz; y pass: j < ny; x pass: i < nx).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "ss3d_bodies.cuh"
#include "ss3d_engine.cuh"
#include "ss3d_internal.h"
#include "ss3d_tma.cuh"

namespace ss3d {

std::atomic<unsigned long long> g_launch_count{0};

constexpr int NT = 256;  // threads per block of every FFT kernel

// tile elements per block: 64 KB of shared memory for the data in both precisions
template <typename R> struct TileE { static constexpr int E = 8192; };
template <> struct TileE<double> { static constexpr int E = 4096; };

template <typename R, int LOGN> struct AxisTX {
  static constexpr int v0 = TileE<R>::E >> LOGN;
  static constexpr int TX = v0 > 64 ? 64 : (v0 < 2 ? 2 : v0);
};
template <typename R, int LOGN> struct RowTX {
  static constexpr int v0 = TileE<R>::E >> LOGN;
  static constexpr int TX = v0 > 64 ? 64 : (v0 < 1 ? 1 : v0);
};

// copy the first cnt entries of the twiddle table of length n into shared memory
template <typename C>
__device__ __forceinline__ void load_tw(C* s, const C* g, int n, int cnt) {
  const C* src = g + (n - 1);
  for (int q = threadIdx.x; q < cnt; q += blockDim.x) s[q] = src[q];
}

// run-time choice of the variant per kernel kind, precision and length
// (kind 0: column pass, 1: column pass with synthesis, 2: C2R rows)
int g_variant[3][2][16] = {};

// Tile configuration of a column pass: variants 0-3 one line per thread
// (ColCfg), 4-7 two lines per thread (PairCfg, FP32 only).
// LPT lines per tile, EB bytes per shared-memory entry.
template <typename R, int LOGN, int V, bool PAIR = (V >= 4)> struct AxisCfg : ColCfg<R, LOGN, V> {
  static constexpr int LPT = ColCfg<R, LOGN, V>::TX;
  static constexpr int EB = sizeof(cpx_t<R>);
};
template <typename R, int LOGN, int V> struct AxisCfg<R, LOGN, V, true> : PairCfg<LOGN, V & 3> {
  static_assert(sizeof(R) == 4, "two-line tiles are FP32 only");
  static constexpr int LPT = 2 * PairCfg<LOGN, V & 3>::TX;
  static constexpr int EB = sizeof(cpair);
};

// c2c transform along a strided axis (in place allowed), unscaled, pruned store.
// FP32 tiles of lengths up to 512 with 8 elements (or pairs) per thread are
// held to 64 registers (two 512-thread CTAs per SM).
template <typename R, int LOGN, int V>
constexpr int col_min_blocks() {
  return (sizeof(R) == 4 && LOGN <= 9 && (V < 4 || (V & 1) == 0) && AxisCfg<R, LOGN, V>::NTH <= 1024)
             ? 1024 / AxisCfg<R, LOGN, V>::NTH
             : 1;
}
// HALF: every kept output position lies below N/2 (a.nout <= N/2)
template <typename R, int LOGN, int SIGN, int V, bool HALF = false>
__global__ void __launch_bounds__(AxisCfg<R, LOGN, V>::NTH, (col_min_blocks<R, LOGN, V>()))
    k_col(AxisArgs a, Geo g, const cpx_t<R>* in, cpx_t<R>* out, Tw tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  using CF = AxisCfg<R, LOGN, V>;
  if constexpr (V >= 4)
    col_body_pair<LOGN, CF::TX, CF::TPC, SIGN, HALF>(a, g, in, out, tw, blockIdx.x, smraw);
  else
    col_body<R, LOGN, CF::TX, CF::TPC, SIGN, HALF>(a, g, in, out, tw, blockIdx.x, smraw);
}

// ---------------------------------------------------------------- middle pass fed by bulk tensor copies
// Variants 8 (one line per thread) and 9 (two lines per thread as a cpair) of
// the FP32 middle (y) pass.  A persistent CTA per SM walks the tiles of the
// pass (LPT consecutive lines x N positions, 64 KB for N >= 128) in the item
// order of col_body.  Tiles are staged by cp.async.bulk.tensor copies into two
// shared-memory stages: while tile q is transformed from stage b, the copy of
// the CTA's next tile lands in stage b ^ 1.  The first radix pass reads its
// inputs from the stage, which then serves as the exchange buffer of the
// later passes; the last pass stores the pruned outputs to global memory as
// col_body does.  The butterflies are those of col_body / col_body_pair, so
// the results are the same bits.
__device__ int g_pipe_err;   // set when a copy wait of a pipelined kernel timed out

template <int LOGN, int P> struct TmaCfg;
template <int LOGN> struct TmaCfg<LOGN, 0> {
  using CF = ColCfg<float, LOGN, 0>;
  using C = float2;
  static constexpr int N = CF::N, TX = CF::TX, TPC = CF::TPC, NTH = CF::NTH, LPT = CF::TX;
};
template <int LOGN> struct TmaCfg<LOGN, 1> {
  using CF = PairCfg<LOGN, 0>;
  using C = cpair;
  static constexpr int N = CF::N, TX = CF::TX, TPC = CF::TPC, NTH = CF::NTH, LPT = 2 * CF::TX;
};
template <int LOGN, int P> struct TmaLayout : TmaCfg<LOGN, P> {
  using B = TmaCfg<LOGN, P>;
  static constexpr int ROWS = B::N < 256 ? B::N : 256;   // rows per copy (a box dimension is at most 256)
  static constexpr int NBOX = B::N / ROWS;
  static constexpr int STAGE = B::N * B::LPT * 8;        // bytes of one staged tile (= its exchange buffer)
  static constexpr int TW_OFF = 2 * STAGE;
  static constexpr int BAR_OFF = TW_OFF + B::N * (int)sizeof(typename B::C);
  static constexpr size_t SMEM = BAR_OFF + 16 + 128;   // + room to align the stages on 128 bytes
  static_assert(B::LPT * 8 % 16 == 0 && B::LPT <= 256, "box rows of whole 16-byte units, at most 256 elements");
  static_assert(STAGE % 128 == 0, "stages on 128-byte boundaries");
};

template <int LOGN, int P>
__global__ void __launch_bounds__(TmaCfg<LOGN, P>::NTH, 1)
    k_col_tma(AxisArgs a, Geo g, float2* out, Tw tw, const __grid_constant__ CUtensorMap map, int ntiles) {
  using L = TmaLayout<LOGN, P>;
  using C = typename L::C;
  constexpr int N = L::N, TX = L::TX, TPC = L::TPC, NTH = L::NTH, LPT = L::LPT;
  constexpr int NR0 = N / Sched<LOGN>::radix(0);
  extern __shared__ __align__(16) unsigned char smdyn[];
  // bulk copies land on 128-byte boundaries: round the dynamic base up
  unsigned char* smraw = smdyn + ((128u - (smem_addr(smdyn) & 127u)) & 127u);
  C* stw = reinterpret_cast<C*>(smraw + L::TW_OFF);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw + L::BAR_OFF);
  const int tid = threadIdx.x;
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  if constexpr (P == 1) {
    load_tw_pair<N, NTH>(reinterpret_cast<cpair*>(stw), tw);
  } else {
    for (int q = tid; q < N; q += NTH) stw[q] = tw.f[N - 1 + q];
  }
  __syncthreads();
  // tile q: realization r, group grp, first line line0 (the item order of col_body)
  auto decode = [&](int q, int& r, int& grp, int& line0) {
    r = q % a.nreal;
    const int tt = q / a.nreal;
    grp = tt / a.tpg;
    line0 = (tt % a.tpg) * LPT;
  };
  auto issue = [&](int q, int b) {   // one thread: arm stage b's barrier and start the copies
    int r, grp, line0;
    decode(q, r, grp, line0);
    unsigned char* dst = smraw + b * L::STAGE;
    mbar_arrive_expect_tx(&bar[b], (uint32_t)L::STAGE);
#pragma unroll
    for (int k = 0; k < L::NBOX; ++k)
      tma_load_3d(dst + k * L::ROWS * LPT * 8, &map, &bar[b], line0, k * L::ROWS, r * a.ngroups + grp);
  };
  int q = blockIdx.x;
  if (tid == 0 && q < ntiles) issue(q, 0);
  const int t = tid % TX;
  const int S = (int)a.S;
  const int nout = a.nout;
  for (int it = 0; q < ntiles; q += gridDim.x, ++it) {
    const int b = it & 1;
    const uint32_t parity = (uint32_t)((it >> 1) & 1);
    const bool ok = mbar_wait_bounded(&bar[b], parity);
    if (__syncthreads_or(!ok)) {
      // a copy did not arrive in time: report it, give it a bounded time to
      // land in this CTA's shared memory, and stop
      if (tid == 0) atomicExch(&g_pipe_err, 1);
      mbar_wait_bounded(&bar[b], parity);
      return;
    }
    if (tid == 0 && q + (int)gridDim.x < ntiles) issue(q + (int)gridDim.x, b ^ 1);
    int r, grp, line0;
    decode(q, r, grp, line0);
    C* s = reinterpret_cast<C*>(smraw + b * L::STAGE);
    if constexpr (P == 0) {
      const bool valid = line_valid(g, line0 + t, a.lines);
      float2* dst = out + ((long long)grp * a.gstride + line0 + t + (long long)r * a.rstride);
      const float2* src = reinterpret_cast<const float2*>(s) + t;
      fft_tile<LOGN, TX, TPC, +1, TX, true, false>(
          s, stw, [&](int jb, int rr) { return src[(jb + rr * NR0) * TX]; },
          [&](int pos, float2 v) {
            if (valid && pos < nout) dst[pos * S] = v;
          });
    } else {
      const int line = line0 + 2 * t;
      const bool valid = line_valid(g, line, a.lines);
      float4* dst = reinterpret_cast<float4*>(out + ((long long)grp * a.gstride + line + (long long)r * a.rstride));
      const float4* src = reinterpret_cast<const float4*>(s) + t;
      const int S2 = S / 2;
      fft_tile<LOGN, TX, TPC, +1, TX, true, false>(
          s, stw, [&](int jb, int rr) { return pair_of(src[(jb + rr * NR0) * TX]); },
          [&](int pos, cpair v) {
            if (valid && pos < nout) dst[pos * S2] = quad_of(v);
          });
    }
    // the stage is refilled by a copy two tiles later: order this tile's
    // shared-memory accesses before it
    fence_proxy_async_smem();
    __syncthreads();
  }
}

// ---------------------------------------------------------------- middle and row passes fused over a cluster
// Row pass variant 5 (FP32, float output, no statistics): the middle (y)
// inverse pass and the C2R row (x) pass of one plane k of one realization in
// one thread-block cluster of CL CTAs, so that the y pass output never goes
// to HBM.  Phase 1: CTA c of the cluster transforms the column tiles
// c, c + CL, ... of the plane along y (TXY columns x NY positions, the tile
// staged from HBM through registers as col_body does) and stores each output
// row j < ny straight into the shared-memory row tile of the CTA that owns
// row j (rows c' TXR .. c' TXR + TXR - 1 belong to CTA c'), through
// distributed shared memory.  A cluster barrier.  Phase 2: each CTA packs,
// transforms and crops its TXR rows exactly as rows_body does after its
// staging, and stores them.  Every column and row sees the butterflies of
// col_body and rows_body, so the results are the same bits.
template <int LY, int LX> struct YXCfg {
  static constexpr int NY = 1 << LY, NX = 1 << LX;
  static constexpr int NTH = 512;
  static constexpr int ETY = 8;                       // phase 1: elements per thread
  static constexpr int TPCY = NY / ETY;
  static constexpr int TXY = NTH / TPCY;              // columns per y tile
  using RC = RowCfg<float, LX, 0>;                    // phase 2: the row tile of rows_body
  static constexpr int TXR = RC::TX, TPCR = RC::TPC, PR = TXR + 1;
  static constexpr bool ok = LY >= 6 && LY <= 9 && LX >= 7 && LX <= 9 && RC::NTH0 == NTH && TXY >= 1 &&
                             TXY <= 64 && TXY * TPCY == NTH;
  static constexpr int ROWBUF = (NX + 1) * PR;        // float2: this CTA's rows, [position][row]
  static constexpr int YP = NY + 4;                   // column pitch of a finished y tile
  static constexpr int YTILE = TXY * YP;              // float2: exchange buffer, then the finished tile
  static constexpr size_t SMEM = (size_t)(ROWBUF + YTILE + NY + 3 * NX) * sizeof(float2);
};

template <int LY, int LX, int CL>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(512, 2)
    k_yx_fused(Geo g, const float2* __restrict__ work, long long wstride, float* __restrict__ out, Tw tw) {
  namespace cg = cooperative_groups;
  using Y = YXCfg<LY, LX>;
  using C = float2;
  constexpr int NY = Y::NY, NX = Y::NX, TXY = Y::TXY, TPCY = Y::TPCY, TXR = Y::TXR, TPCR = Y::TPCR, PR = Y::PR;
  constexpr int NTH = Y::NTH;
  constexpr int NR0 = NY / Sched<LY>::radix(0);
  extern __shared__ __align__(16) unsigned char smraw[];
  C* rowbuf = reinterpret_cast<C*>(smraw);
  C* ytile = rowbuf + Y::ROWBUF;
  C* stwy = ytile + Y::YTILE;   // NY entries e^{-2 pi i m/NY}
  C* stw = stwy + NY;           // 2 NX entries e^{-2 pi i m/(2 NX)}
  C* stwN = stw + 2 * NX;       // NX entries e^{-2 pi i m/NX}
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int plane = blockIdx.x / CL;   // r nz + k
  const int r = plane / g.nz, k = plane - (plane / g.nz) * g.nz;
  const int tid = threadIdx.x;
  for (int q = tid; q < NY; q += NTH) stwy[q] = tw.f[NY - 1 + q];
  for (int q = tid; q < 2 * NX; q += NTH) stw[q] = tw.f[2 * NX - 1 + q];
  for (int q = tid; q < NX; q += NTH) stwN[q] = tw.f[NX - 1 + q];
  // every CTA of the cluster has started (its shared memory exists) before any
  // CTA writes into it
  cl.sync();
  // ---- phase 1: y transforms of this CTA's column tiles, rows j < ny to their owners
  const C* pin = work + (long long)r * wstride + (long long)k * g.npy * g.HP;
  const int H = g.H;
  const int ntiles = (H + TXY - 1) / TXY;
  const int t = tid % TXY;
  const int S = g.HP;
  const int ny = g.ny;
  constexpr int YP = Y::YP;
  for (int u = rank; u < ntiles; u += CL) {
    const int i = u * TXY + t;
    const bool valid = i < H;
    const C* src = pin + (valid ? i : 0);
    // the finished tile goes to shared memory column by column (pitch NY + 4:
    // the 8 columns x 4 consecutive positions of a warp's store hit every bank
    // pair twice) ...
    fft_tile<LY, TXY, TPCY, +1, TXY, false, true>(
        ytile, stwy, [&](int jb, int rr) { return src[(jb + rr * NR0) * S]; },
        [&](int pos, C v) { ytile[t * YP + pos] = v; });
    __syncthreads();
    // ... and from there to the owners of its rows, a warp storing consecutive
    // positions of one column (contiguous in the owner's row tile)
    const int ncol = min(TXY, H - u * TXY);
    for (int q = tid; q < ncol * ny; q += NTH) {
      const int cc = q / ny, pos = q - cc * ny;
      const int owner = pos / TXR;
      C* rb = cl.map_shared_rank(rowbuf, owner);
      rb[(u * TXY + cc) * PR + (pos - owner * TXR)] = ytile[cc * YP + pos];
    }
    __syncthreads();   // the next tile reuses the buffer
  }
  cl.sync();           // every row tile of the cluster is complete
  // ---- phase 2: C2R of rows j = rank TXR + tt (the steps of rows_body after its staging)
  for (int q = tid; q < (NX / 2 + 1) * TXR; q += NTH) {
    const int tt = q % TXR, kk = q / TXR;
    const int kc = NX - kk;
    C a = rowbuf[kk * PR + tt], b = rowbuf[kc * PR + tt];
    if (kk == 0) {
      a.y = 0.f;
      b.y = 0.f;
    }
    C w = stw[kk];
    w.y = -w.y;
    const C bc = cmk<C>(b.x, -b.y);
    const C zk = cadd(cadd(a, bc), cmul_si<+1>(cmul(w, csub(a, bc))));
    if (kk != 0 && kc != kk) {
      C w2 = stw[kc];
      w2.y = -w2.y;
      const C ac = cmk<C>(a.x, -a.y);
      rowbuf[kc * PR + tt] = cadd(cadd(b, ac), cmul_si<+1>(cmul(w2, csub(b, ac))));
    }
    rowbuf[kk * PR + tt] = zk;
  }
  __syncthreads();
  fft_rows_inv<float, LX, TXR, TPCR>(rowbuf, stwN);
  float* dst = out + (long long)r * ((long long)g.nx * g.ny * g.nz) + (long long)k * g.ny * g.nx;
  const int nxh = (g.nx + 1) / 2;
  const bool even = (g.nx & 1) == 0;
  const int lane = tid & 31, warp = tid >> 5;
  for (int tt = warp; tt < TXR; tt += NTH / 32) {
    const int j = rank * TXR + tt;
    if (j >= ny) break;
    float* rp = dst + (long long)j * g.nx;
    for (int m = lane; m < nxh; m += 32) {
      const C z = rowbuf[m * PR + tt];
      if (even) {
        reinterpret_cast<float2*>(rp)[m] = make_float2(z.x, z.y);
      } else {
        rp[2 * m] = z.x;
        if (2 * m + 1 < g.nx) rp[2 * m + 1] = z.y;
      }
    }
  }
}

// first inverse pass with the coefficient synthesis fused into the loader
// (GAUSS: igauss of the realizations, 0 phases, 1 Gaussian coefficients;
// HALF: every kept output position lies below N/2)
template <typename R, int LOGN, int V, int GAUSS, bool HALF = false>
__global__ void __launch_bounds__(AxisCfg<R, LOGN, V>::NTH) k_colgen(AxisArgs a, Geo g, const R* __restrict__ amp,
                                                                    const uint32_t* __restrict__ rowstates,
                                                                    const uint32_t* __restrict__ apow,
                                                                    cpx_t<R>* out, Tw tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  using CF = AxisCfg<R, LOGN, V>;
  if constexpr (V >= 4)
    colgen_body_pair<LOGN, CF::TX, CF::TPC, GAUSS, HALF>(a, g, amp, rowstates, apow, out, tw, blockIdx.x, smraw);
  else
    colgen_body<R, LOGN, CF::TX, CF::TPC, GAUSS, HALF>(a, g, amp, rowstates, apow, out, tw, blockIdx.x, smraw);
}

// Standalone synthesis of the full half spectrum of nreal realizations.
template <typename R>
__global__ void k_gen(Geo g, const R* __restrict__ amp, const uint32_t* __restrict__ rowstates,
                      const uint32_t* __restrict__ apow, cpx_t<R>* out, long long rstride, int nreal) {
  using C = cpx_t<R>;
  const long long per = (long long)g.npz * g.npy * g.HP;
  const long long tot = per * nreal;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
       q += (long long)gridDim.x * blockDim.x) {
    int r = (int)(q / per);
    long long o = q - r * per;
    int i = (int)(o % g.HP);
    long long rest = o / g.HP;
    int j = (int)(rest % g.npy), k = (int)(rest / g.npy);
    C v = cmk<C>(R(0), R(0));
    if (i < g.H) v = coefficient<R>(g, i, j, k, amp[o], rowstates + (size_t)r * g.npy * g.npz, apow);
    out[o + r * rstride] = v;
  }
}

// State of the first draw of every row of every realization of the batch:
// s = 16807^(11 + (r_first + r) * D + d * prefix(row)) * s0  (mod 2^31-1).
// Layout [r][j][k] (k fastest): the first inverse pass runs along k, so the
// rows a warp needs are contiguous.
__global__ void k_rowstates(Geo g, uint32_t s0, long long r_first, int nreal, const uint32_t* __restrict__ ptab,
                            uint32_t* rowstates) {
  const int rows = g.npy * g.npz;
  const long long tot = (long long)rows * nreal;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
       q += (long long)gridDim.x * blockDim.x) {
    int r = (int)(q / rows);
    int row = (int)(q - (long long)r * rows);
    int j = row / g.npz, k = row % g.npz;
    const uint64_t M1 = (uint64_t)(PM_M - 1);
    uint64_t t = ((uint64_t)(r_first + r) % M1) * (g.D % M1) % M1;
    t = (t + (uint64_t)g.d * row_prefix(g, j, k)) % M1;
    rowstates[q] = pm_mulmod(pm_pow(ptab, 11ull + t), s0);
  }
}

// a^(d*i) mod m for i in [0, npx): the offset of index i inside a row
__global__ void k_apow(int npx, int d, const uint32_t* __restrict__ ptab, uint32_t* apow) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += gridDim.x * blockDim.x)
    apow[i] = pm_pow(ptab, (uint64_t)d * i);
}

// First-draw state of every half-spectrum index of one realization (test hook)
__global__ void k_debug_states(Geo g, const uint32_t* __restrict__ rs, const uint32_t* __restrict__ apow,
                               uint32_t* out) {
  const long long tot = (long long)g.npz * g.npy * g.H;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
       q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % g.H);
    long long row = q / g.H;
    int j = (int)(row % g.npy), k = (int)(row / g.npy);
    bool conj, self;
    out[q] = first_state(g, i, j, k, rs, apow, conj, self);
  }
}

// ---------------------------------------------------------------- x pass: C2R + crop
template <typename R, typename O, int LOGN, int V>
__global__ void __launch_bounds__(RowCfg<R, LOGN, V>::NTH) k_rows_c2r(Geo g, const cpx_t<R>* __restrict__ in,
                                                                      long long rstride, O* __restrict__ out,
                                                                      long long ostride, int nreal, int nblk_per_r,
                                                                      double* __restrict__ part, Tw tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  using RC = RowCfg<R, LOGN, V>;
  static_assert(RC::NTH == RC::TX * RC::TPC, "row tile of whole warps");
  rows_body<R, O, LOGN, RC::TX, RC::TPC>(g, in, rstride, out, ostride, nreal, nblk_per_r, part, tw, blockIdx.x,
                                         smraw);
}

// x pass with the rows held in warps (rows_warp_body); HALF: the crop keeps
// at most the first N/2 complex values of each packed row ((nx + 1)/2 <= N/2)
template <typename R, typename O, int LOGN, bool HALF = false>
__global__ void __launch_bounds__(RowWarpCfg<R, LOGN>::NTH)
    k_rows_warp(Geo g, const cpx_t<R>* __restrict__ in, long long rstride, O* __restrict__ out, long long ostride,
                int nreal, int nblk_per_r, double* __restrict__ part, Tw tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  rows_warp_body<R, O, LOGN, HALF>(g, in, rstride, out, ostride, nreal, nblk_per_r, part, tw, blockIdx.x, smraw);
}

// x pass with two rows per lane on packed FP32 (rows_pair_body)
template <typename O, int LOGN>
__global__ void __launch_bounds__(RowPairCfg<LOGN>::NTH, 3)
    k_rows_pair(Geo g, const float2* __restrict__ in, long long rstride, O* __restrict__ out, long long ostride,
                int nreal, int nblk_per_r, double* __restrict__ part, Tw tw) {
  extern __shared__ __align__(16) unsigned char smraw[];
  rows_pair_body<O, LOGN>(g, in, rstride, out, ostride, nreal, nblk_per_r, part, tw, blockIdx.x, smraw);
}

// npx == 1: the x axis is trivial, x[0] = Re X[0]
template <typename R, typename O>
__global__ void k_rows_copy(Geo g, const cpx_t<R>* __restrict__ in, long long rstride, O* __restrict__ out,
                            long long ostride, int nreal, int nblk_per_r, double* __restrict__ part) {
  const int r = blockIdx.x % nreal;
  const int blk = blockIdx.x / nreal;
  const int nrows = g.ny * g.nz;
  double s1 = 0, s2 = 0;
  int row = blk * NT + threadIdx.x;
  if (row < nrows) {
    int j = row % g.ny, k = row / g.ny;
    R v = in[(long long)r * rstride + ((long long)k * g.npy + j) * g.HP].x;
    out[(long long)r * ostride + row] = (O)v;
    s1 = v;
    s2 = (double)v * v;
  }
  if (part) {
    block_sum2<NT>(s1, s2);
    if (threadIdx.x == 0) {
      part[2 * ((long long)r * nblk_per_r + blk)] = s1;
      part[2 * ((long long)r * nblk_per_r + blk) + 1] = s2;
    }
  }
}

__global__ void k_reduce_zstats(const double* __restrict__ part, int nblk, double* zsum) {
  const int r = blockIdx.x;
  double a = 0, b = 0;
  for (int q = threadIdx.x; q < nblk; q += NT) {
    a += part[2 * ((long long)r * nblk + q)];
    b += part[2 * ((long long)r * nblk + q) + 1];
  }
  block_sum2<NT>(a, b);
  if (threadIdx.x == 0) {
    zsum[2 * r] = a;
    zsum[2 * r + 1] = b;
  }
}

// ---------------------------------------------------------------- spectrum
// x pass of the forward transform with the covariance grid generated in place
// (f90:1256-1270): row (j,k) of c(i,j,k) = C(ip dx, jp dy, kp dz) with minimum
// image lags, R2C of length npx = 2N through a length-N complex FFT:
//   X[q] = (Z[q] + conj Z[N-q])/2 - i/2 w^q (Z[q] - conj Z[N-q]),  w = e^{-2 pi i/(2N)}
// C at the lag whose range-scaled rotated components are b + ip s per
// structure (b: the row's lag (0, jp dy, kp dz), s: one x step, both rotated
// and divided by the range): the covariance of f90:153-178 with the rotation
// of a row done once, no division per point, and for the gaussian model no
// square root (it needs only h^2)
__device__ __forceinline__ double cov_row_point(const Model& m, const double* __restrict__ b,
                                                const double* __restrict__ sx, double ip, bool origin) {
  double c = origin ? m.nugget : 0.0;
  for (int st = 0; st < m.nst; st++) {
    const double rx = fma(ip, sx[3 * st], b[3 * st]);
    const double ry = fma(ip, sx[3 * st + 1], b[3 * st + 1]);
    const double rz = fma(ip, sx[3 * st + 2], b[3 * st + 2]);
    const double h2 = rx * rx + ry * ry + rz * rz;
    if (m.itype[st] == 1) {
      const double hr = sqrt(h2);
      if (hr < 1.0) c = c + m.sill[st] * (1.0 - 1.5 * hr + 0.5 * (hr * hr * hr));
    } else if (m.itype[st] == 2) {
      c = c + m.sill[st] * exp(-3.0 * sqrt(h2));
    } else {
      c = c + m.sill[st] * exp(-(3.0 * h2));
    }
  }
  return c;
}

template <int LOGN>
__global__ void __launch_bounds__(NT) k_spec_rows(Model m, double dx, double dy, double dz, Geo g,
                                                  double2* __restrict__ out, Tw tw) {
  using C = double2;
  constexpr int N = 1 << LOGN;
  constexpr int TX = RowTX<double, LOGN>::TX;
  constexpr int PITCH = TX + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  C* stw = s + (N + 1) * PITCH;
  const int nrows = g.npy * g.npz;
  const int row0 = blockIdx.x * TX;
  double* rb = reinterpret_cast<double*>(stw + 2 * N);   // [TX][MAXST][3] rotated row lags / range
  double* rsx = rb + TX * MAXST * 3;                      // [MAXST][3] rotated x step / range
  load_tw(stw, tw.d, 2 * N, 2 * N);
  for (int q = threadIdx.x; q < (TX + 1) * m.nst; q += NT) {
    const int t = q / m.nst, st = q - t * m.nst;
    const double* r = m.rot[st];
    const double ia = 1.0 / m.ahmax[st];
    if (t == TX) {
      for (int c = 0; c < 3; c++) rsx[3 * st + c] = r[3 * c] * dx * ia;
    } else {
      const int row = min(row0 + t, nrows - 1);
      const int j = row % g.npy, k = row / g.npy;
      const double y = (double)(j > g.npy / 2 ? j - g.npy : j) * dy;
      const double z = (double)(k > g.npz / 2 ? k - g.npz : k) * dz;
      for (int c = 0; c < 3; c++) rb[(t * MAXST + st) * 3 + c] = (r[3 * c + 1] * y + r[3 * c + 2] * z) * ia;
    }
  }
  __syncthreads();
  for (int q = threadIdx.x; q < N * TX; q += NT) {
    int t = q / N, p = q % N;
    int row = row0 + t;
    C v = cmk<C>(0.0, 0.0);
    if (row < nrows) {
      const int j = row % g.npy, k = row / g.npy;
      const bool jk0 = j == 0 && k == 0;
      int i0 = 2 * p, i1 = 2 * p + 1;
      int ip0 = i0 > g.npx / 2 ? i0 - g.npx : i0;
      int ip1 = i1 > g.npx / 2 ? i1 - g.npx : i1;
      const double* b = rb + t * MAXST * 3;
      v.x = cov_row_point(m, b, rsx, (double)ip0, jk0 && ip0 == 0);
      v.y = cov_row_point(m, b, rsx, (double)ip1, jk0 && ip1 == 0);
    }
    s[p * PITCH + t] = v;
  }
  __syncthreads();
  smem_fft<LOGN, TX, PITCH, NT, -1, 2>(s, stw);
  for (int q = threadIdx.x; q < (N / 2 + 1) * TX; q += NT) {
    int t = q % TX, k = q / TX;
    int kc = N - k;
    C zk = s[k * PITCH + t];
    C zc = s[(kc % N) * PITCH + t];
    C zcc = cmk<C>(zc.x, -zc.y), zkc = cmk<C>(zk.x, -zk.y);
    C w = stw[k];
    C sum = cadd(zk, zcc), dif = csub(zk, zcc);
    C xk = cmk<C>(0.5 * sum.x, 0.5 * sum.y);
    C wd = cmul(w, dif);
    xk = cadd(xk, cmk<C>(0.5 * wd.y, -0.5 * wd.x));   // - i/2 * w * dif
    if (kc != k) {
      C w2 = stw[kc];   // kc <= N < 2N entries
      C sum2 = cadd(zc, zkc), dif2 = csub(zc, zkc);
      C wd2 = cmul(w2, dif2);
      C xc = cadd(cmk<C>(0.5 * sum2.x, 0.5 * sum2.y), cmk<C>(0.5 * wd2.y, -0.5 * wd2.x));
      s[kc * PITCH + t] = xc;
    }
    s[k * PITCH + t] = xk;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < (N + 1) * TX; q += NT) {
    int t = q / (N + 1), p = q % (N + 1);
    int row = row0 + t;
    if (row < nrows) {
      int j = row % g.npy, k = row / g.npy;
      out[((long long)k * g.npy + j) * g.HP + p] = s[p * PITCH + t];
    }
  }
}

// The same rows (covariance and R2C) with each row in the registers of the
// TPC lanes of one warp, for N = npx/2 <= 256 (8 complex values per lane):
// a lane computes its 16 covariance values (the real pairs at x = 2q, 2q + 1)
// straight into the registers of the first radix pass, the register engine
// transforms them on the warp's shared slice, the transform is staged once in
// that slice in natural order, and the split reads Z[k] and Z[N-k] and stores
// X[k] and X[N-k] of the row (k <= N/2).  The shared-memory row tile of
// k_spec_rows also stages the input, runs every radix pass through shared
// memory and splits in place.
template <int LOGN> struct SpecWarpCfg {
  static constexpr int N = 1 << LOGN;
  static constexpr int ET = 8;                  // complex values per lane
  static constexpr int TPC = N / ET;            // lanes per row
  static constexpr int RPW = TPC >= 32 ? 1 : 32 / TPC;
  static constexpr int NW = 8;                  // warps per block
  static constexpr int NTH = 32 * NW;
  static constexpr int ROWS = NW * RPW;         // rows per block
  static constexpr int SLICE = N * RPW;         // exchange elements per warp
  static constexpr bool ok = LOGN >= 3 && LOGN <= 8;
  static constexpr size_t smem =
      (size_t)(3 * N + NW * SLICE) * sizeof(double2) + (size_t)(ROWS + 1) * MAXST * 3 * sizeof(double);
};

template <int LOGN>
__global__ void __launch_bounds__(SpecWarpCfg<LOGN>::NTH) k_spec_rows_warp(Model m, double dx, double dy, double dz,
                                                                          Geo g, double2* __restrict__ out, Tw tw) {
  using C = double2;
  using W = SpecWarpCfg<LOGN>;
  constexpr int N = W::N, ET = W::ET, TPC = W::TPC, RPW = W::RPW;
  static_assert(W::ok && TPC * RPW == 32, "rows of whole warps");
  extern __shared__ __align__(16) unsigned char smraw[];
  C* stw = reinterpret_cast<C*>(smraw);   // 2N entries e^{-2 pi i m/(2N)} (the split)
  C* stwN = stw + 2 * N;                  // N entries e^{-2 pi i m/N} (the transform)
  C* slices = stwN + N;
  double* rb = reinterpret_cast<double*>(slices + W::NW * W::SLICE);   // [ROWS][MAXST][3]
  double* rsx = rb + W::ROWS * MAXST * 3;                             // [MAXST][3]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  C* sx = slices + warp * W::SLICE;
  const int nrows = g.npy * g.npz;
  const int rowb = blockIdx.x * W::ROWS;
  for (int q = threadIdx.x; q < 2 * N; q += W::NTH) stw[q] = tw.d[2 * N - 1 + q];
  for (int q = threadIdx.x; q < N; q += W::NTH) stwN[q] = tw.d[N - 1 + q];
  for (int q = threadIdx.x; q < (W::ROWS + 1) * m.nst; q += W::NTH) {
    const int t = q / m.nst, st = q - t * m.nst;
    const double* r = m.rot[st];
    const double ia = 1.0 / m.ahmax[st];
    if (t == W::ROWS) {
      for (int cc = 0; cc < 3; cc++) rsx[3 * st + cc] = r[3 * cc] * dx * ia;
    } else {
      const int row = min(rowb + t, nrows - 1);
      const int j = row % g.npy, k = row / g.npy;
      const double y = (double)(j > g.npy / 2 ? j - g.npy : j) * dy;
      const double z = (double)(k > g.npz / 2 ? k - g.npz : k) * dz;
      for (int cc = 0; cc < 3; cc++) rb[(t * MAXST + st) * 3 + cc] = (r[3 * cc + 1] * y + r[3 * cc + 2] * z) * ia;
    }
  }
  __syncthreads();
  const int t = lane % RPW, c = lane / RPW;
  const int rw = warp * RPW + t;
  const int row = rowb + rw;
  const bool ok = row < nrows;
  const int j = ok ? row % g.npy : 0, k = ok ? row / g.npy : 0;
  const bool jk0 = j == 0 && k == 0;
  const double* b = rb + rw * MAXST * 3;
  constexpr int R0 = Sched<LOGN>::radix(0), NBT = ET / R0;
  C v[ET];
  // pass-0 order of the engine: v[mm R0 + r] holds position c + TPC mm + r N / R0
#pragma unroll
  for (int mm = 0; mm < NBT; ++mm)
#pragma unroll
    for (int r = 0; r < R0; ++r) {
      const int q = c + TPC * mm + r * (N / R0);
      const int i0 = 2 * q, i1 = 2 * q + 1;
      const int ip0 = i0 > g.npx / 2 ? i0 - g.npx : i0;
      const int ip1 = i1 > g.npx / 2 ? i1 - g.npx : i1;
      C zv = cmk<C>(0.0, 0.0);
      if (ok) {
        zv.x = cov_row_point(m, b, rsx, (double)ip0, jk0 && ip0 == 0);
        zv.y = cov_row_point(m, b, rsx, (double)ip1, jk0 && ip1 == 0);
      }
      v[mm * R0 + r] = zv;
    }
  fft_tile_regs<LOGN, RPW, TPC, -1, RPW, false, true, -1>(
      sx, stwN, v, t, c, [&](int pos, C zz) { sx[xidx<RPW, -1>(pos, t)] = zz; });
  __syncwarp();
  if (ok) {
    C* orow = out + ((long long)k * g.npy + j) * g.HP;
    for (int kk = c; kk <= N / 2; kk += TPC) {
      const int kc = N - kk;
      const C zk = sx[xidx<RPW, -1>(kk, t)];
      const C zc = sx[xidx<RPW, -1>(kc & (N - 1), t)];
      const C zcc = cmk<C>(zc.x, -zc.y), zkc = cmk<C>(zk.x, -zk.y);
      const C w = stw[kk];
      const C sum = cadd(zk, zcc), dif = csub(zk, zcc);
      const C wd = cmul(w, dif);
      orow[kk] = cadd(cmk<C>(0.5 * sum.x, 0.5 * sum.y), cmk<C>(0.5 * wd.y, -0.5 * wd.x));   // - i/2 w dif
      if (kc != kk) {
        const C w2 = stw[kc];
        const C sum2 = cadd(zc, zkc), dif2 = csub(zc, zkc);
        const C wd2 = cmul(w2, dif2);
        orow[kc] = cadd(cmk<C>(0.5 * sum2.x, 0.5 * sum2.y), cmk<C>(0.5 * wd2.y, -0.5 * wd2.x));
      }
    }
  }
}

// c2c transform of nrows contiguous rows of length 2^LOGN in place, unscaled
// (the x pass of the full-grid transform ss3d_fft3d): TX rows staged in
// shared memory, the shared-memory Stockham engine, rows written back
template <int LOGN, int SIGN>
__global__ void __launch_bounds__(NT) k_rows_c2c(long long nrows, double2* __restrict__ a, Tw tw) {
  using C = double2;
  constexpr int N = 1 << LOGN;
  constexpr int TX = RowTX<double, LOGN>::TX;
  constexpr int PITCH = TX + 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  C* stw = s + N * PITCH;
  const long long row0 = (long long)blockIdx.x * TX;
  load_tw(stw, tw.d, N, N);
  for (int q = threadIdx.x; q < N * TX; q += NT) {
    const int t = q / N, p = q % N;
    const long long row = row0 + t;
    s[p * PITCH + t] = row < nrows ? a[row * N + p] : cmk<C>(0.0, 0.0);
  }
  __syncthreads();
  smem_fft<LOGN, TX, PITCH, NT, SIGN, 1>(s, stw);
  for (int q = threadIdx.x; q < N * TX; q += NT) {
    const int t = q / N, p = q % N;
    const long long row = row0 + t;
    if (row < nrows) a[row * N + p] = s[p * PITCH + t];
  }
}

// npx == 1: X[0] = c(0, j, k)
__global__ void k_spec_rows_n1(Model m, double dx, double dy, double dz, Geo g, double2* __restrict__ out) {
  const int nrows = g.npy * g.npz;
  for (int row = blockIdx.x * blockDim.x + threadIdx.x; row < nrows; row += gridDim.x * blockDim.x) {
    int j = row % g.npy, k = row / g.npy;
    int kp = k > g.npz / 2 ? k - g.npz : k;
    int jp = j > g.npy / 2 ? j - g.npy : j;
    out[(long long)row * g.HP] = make_double2(covariance(m, 0.0 * dx, (double)jp * dy, (double)kp * dz), 0.0);
  }
}

// S = X / ntot, amp = sqrt(max(Re S, 0)), diagnostics over the full spectrum
// (indices 0 < i < npx/2 stand for themselves and their mirror).  f90:1273-1292
__global__ void k_spec_amp(Geo g, const double2* __restrict__ X, double* __restrict__ amp64,
                           float* __restrict__ amp32, SpecPartial* part) {
  const long long tot = (long long)g.npz * g.npy * g.HP;
  // 1/N: N = npx npy npz is a power of two, so the product by its reciprocal
  // is exactly the division X / N of f90:1273-1274
  const double irn = 1.0 / ((double)g.npx * (double)g.npy * (double)g.npz);
  double mi = 0, mr = 0, sp = 0, sn = 0;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < tot;
       q += (long long)gridDim.x * blockDim.x) {
    int i = (int)(q % g.HP);
    double a = 0.0;
    if (i < g.H) {
      double2 v = X[q];
      double re = v.x * irn, im = v.y * irn;
      double w = (i == 0 || 2 * i == g.npx) ? 1.0 : 2.0;
      mi = fmax(mi, fabs(im));
      mr = fmax(mr, fabs(re));
      if (re < 0.0) {
        sn += w * re;
      } else {
        sp += w * re;
        a = sqrt(re);
      }
    }
    if (amp64) amp64[q] = a;
    if (amp32) amp32[q] = (float)a;
  }
  __shared__ double red[4][NT / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    mi = fmax(mi, __shfl_down_sync(0xffffffffu, mi, off));
    mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
    sp += __shfl_down_sync(0xffffffffu, sp, off);
    sn += __shfl_down_sync(0xffffffffu, sn, off);
  }
  if ((threadIdx.x & 31) == 0) {
    int w = threadIdx.x >> 5;
    red[0][w] = mi;
    red[1][w] = mr;
    red[2][w] = sp;
    red[3][w] = sn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    SpecPartial p{0, 0, 0, 0};
    for (int w = 0; w < NT / 32; ++w) {
      p.maximag = fmax(p.maximag, red[0][w]);
      p.maxreal = fmax(p.maxreal, red[1][w]);
      p.spos += red[2][w];
      p.sneg += red[3][w];
    }
    part[blockIdx.x] = p;
  }
}

// Last forward pass (z) of the spectrum with the amplitude step fused into its
// stores (f90:1273-1292): S = X / N, amp = sqrt(max(Re S, 0)) in FP64 and its
// FP32 copy, written straight from the registers of the transform instead of
// storing X and reading it back; the padding columns get amplitude 0.  Per
// block diagnostics (max |Im S|, max |Re S|, sums of the positive and negative
// parts of S over the full spectrum, indices 0 < i < npx/2 counting for
// themselves and their mirror) go to part[blockIdx.x] for k_reduce_spec.
template <int LOGN>
__global__ void __launch_bounds__(ColCfg<double, LOGN, 0>::NTH)
    k_col_amp(AxisArgs a, Geo g, const double2* __restrict__ in, double* __restrict__ amp64, float* __restrict__ amp32,
              Tw tw, SpecPartial* __restrict__ part) {
  using C = double2;
  using CF = ColCfg<double, LOGN, 0>;
  constexpr int N = 1 << LOGN, TX = CF::TX, TPC = CF::TPC, NTH = CF::NTH;
  constexpr int NR0 = N / Sched<LOGN>::radix(0);
  extern __shared__ __align__(16) unsigned char smraw[];
  C* s = reinterpret_cast<C*>(smraw);
  C* stw = s + N * TX;
  const int line0 = blockIdx.x * TX;
  const int t = threadIdx.x % TX;
  const int line = line0 + t;
  const bool inside = line < a.lines;
  const int i = inside ? line % g.HP : 0;
  const bool valid = inside && i < g.H;
  const C* src = in + (valid ? line : 0);
  const int S = (int)a.S;
  // 1/N: N = npx npy npz is a power of two, so the product by its reciprocal
  // is exactly the division X / N of f90:1273-1274
  const double irn = 1.0 / ((double)g.npx * (double)g.npy * (double)g.npz);
  const double wgt = (i == 0 || 2 * i == g.npx) ? 1.0 : 2.0;
  double mi = 0.0, mr = 0.0, sp = 0.0, sn = 0.0;
  for (int q = threadIdx.x; q < N; q += NTH) stw[q] = tw.d[N - 1 + q];
  __syncthreads();
  fft_tile<LOGN, TX, TPC, -1>(
      s, stw, [&](int jb, int r) { return src[(jb + r * NR0) * S]; },
      [&](int pos, C v) {
        if (valid) {
          const double re = v.x * irn, im = v.y * irn;
          mi = fmax(mi, fabs(im));
          mr = fmax(mr, fabs(re));
          double am = 0.0;
          if (re < 0.0) {
            sn += wgt * re;
          } else {
            sp += wgt * re;
            am = sqrt(re);
          }
          amp64[(long long)pos * S + line] = am;
          amp32[(long long)pos * S + line] = (float)am;
        } else if (inside) {
          amp64[(long long)pos * S + line] = 0.0;
          amp32[(long long)pos * S + line] = 0.0f;
        }
      });
  __shared__ double red[4][NTH / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    mi = fmax(mi, __shfl_down_sync(0xffffffffu, mi, off));
    mr = fmax(mr, __shfl_down_sync(0xffffffffu, mr, off));
    sp += __shfl_down_sync(0xffffffffu, sp, off);
    sn += __shfl_down_sync(0xffffffffu, sn, off);
  }
  if ((threadIdx.x & 31) == 0) {
    const int w = threadIdx.x >> 5;
    red[0][w] = mi;
    red[1][w] = mr;
    red[2][w] = sp;
    red[3][w] = sn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    SpecPartial p{0, 0, 0, 0};
    for (int w = 0; w < NTH / 32; ++w) {
      p.maximag = fmax(p.maximag, red[0][w]);
      p.maxreal = fmax(p.maxreal, red[1][w]);
      p.spos += red[2][w];
      p.sneg += red[3][w];
    }
    part[blockIdx.x] = p;
  }
}

// Sum of the per-block partials in a fixed order, independent of scheduling:
// one block of RS_NT threads; thread t combines partials t, t + RS_NT, ... in
// index order, then each warp folds its lanes by halving distances, and warp 0
// folds the warp results the same way.
constexpr int RS_NT = 1024;
__device__ __forceinline__ void spec_combine(SpecPartial& a, const SpecPartial& b) {
  a.maximag = fmax(a.maximag, b.maximag);
  a.maxreal = fmax(a.maxreal, b.maxreal);
  a.spos += b.spos;
  a.sneg += b.sneg;
}
__device__ __forceinline__ void spec_warp_fold(SpecPartial& p) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    SpecPartial o;
    o.maximag = __shfl_down_sync(0xffffffffu, p.maximag, off);
    o.maxreal = __shfl_down_sync(0xffffffffu, p.maxreal, off);
    o.spos = __shfl_down_sync(0xffffffffu, p.spos, off);
    o.sneg = __shfl_down_sync(0xffffffffu, p.sneg, off);
    spec_combine(p, o);
  }
}
__global__ void __launch_bounds__(RS_NT) k_reduce_spec(const SpecPartial* __restrict__ part, int n,
                                                       SpecPartial* out) {
  __shared__ SpecPartial red[RS_NT / 32];
  SpecPartial p{0, 0, 0, 0};
  for (int q = threadIdx.x; q < n; q += RS_NT) spec_combine(p, part[q]);
  spec_warp_fold(p);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = p;
  __syncthreads();
  if (warp == 0) {
    p = red[lane];   // RS_NT / 32 == 32 warp results
    spec_warp_fold(p);
    if (lane == 0) *out = p;
  }
}
static_assert(RS_NT / 32 == 32, "warp 0 folds one result per warp");

// ---------------------------------------------------------------- launch helpers
static int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

template <typename K>
static cudaError_t set_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return func_smem(reinterpret_cast<const void*>(kernel), bytes);
}

#define SS3D_LOGN_SWITCH(LOGN_VAR, MAXL, CALL)                  \
  switch (LOGN_VAR) {                                            \
    case 0: { constexpr int L = 0; if constexpr (L <= MAXL) { CALL; } break; } \
    case 1: { constexpr int L = 1; if constexpr (L <= MAXL) { CALL; } break; } \
    case 2: { constexpr int L = 2; if constexpr (L <= MAXL) { CALL; } break; } \
    case 3: { constexpr int L = 3; if constexpr (L <= MAXL) { CALL; } break; } \
    case 4: { constexpr int L = 4; if constexpr (L <= MAXL) { CALL; } break; } \
    case 5: { constexpr int L = 5; if constexpr (L <= MAXL) { CALL; } break; } \
    case 6: { constexpr int L = 6; if constexpr (L <= MAXL) { CALL; } break; } \
    case 7: { constexpr int L = 7; if constexpr (L <= MAXL) { CALL; } break; } \
    case 8: { constexpr int L = 8; if constexpr (L <= MAXL) { CALL; } break; } \
    case 9: { constexpr int L = 9; if constexpr (L <= MAXL) { CALL; } break; } \
    case 10: { constexpr int L = 10; if constexpr (L <= MAXL) { CALL; } break; } \
    case 11: { constexpr int L = 11; if constexpr (L <= MAXL) { CALL; } break; } \
    case 12: { constexpr int L = 12; if constexpr (L <= MAXL) { CALL; } break; } \
    default: return cudaErrorInvalidValue;                       \
  }

// lengths with pruned (HALF) forms of the inverse passes
constexpr bool half_len(int L) { return L >= 5 && L <= 10; }

template <typename R> struct MaxL { static constexpr int v = MAX_LOGN_F; };
template <> struct MaxL<double> { static constexpr int v = MAX_LOGN_D; };

template <typename R, int L, int SIGN, int V>
static cudaError_t run_axis_c2c_v(const AxisArgs& a, const Geo& g, const cpx_t<R>* in, cpx_t<R>* out, Tw tw,
                                  cudaStream_t st) {
  using CF = AxisCfg<R, L, V>;
  if constexpr (L == 0) {
    // length-1 transform: identity; copy when out-of-place
    if (in != out) return cudaErrorInvalidValue;
    return cudaSuccess;
  } else {
    size_t smem = (size_t)(CF::N * CF::TX + CF::N) * CF::EB;
    auto kern = k_col<R, L, SIGN, V>;
    // pruned inverse passes that keep at most half of the positions (the
    // padded grid is at least twice the simulated one along most axes); the
    // two-line tiles (V >= 4) of 64 positions keep the unpruned form: built
    // pruned, they did not reproduce the bits of the other tiles
    if constexpr (SIGN > 0 && half_len(L) && (V < 4 || L >= 7))
      if (2 * a.nout <= CF::N) kern = k_col<R, L, SIGN, V, true>;
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    AxisArgs b = a;
    b.tpg = (a.lines + CF::LPT - 1) / CF::LPT;
    unsigned blocks = (unsigned)((long long)b.tpg * a.ngroups * a.nreal);
    kern<<<blocks, CF::NTH, smem, st>>>(b, g, in, out, tw);
    ++g_launch_count;
    return cudaGetLastError();
  }
}

// ---- host side of the pipelined middle pass
std::atomic<unsigned long long> g_pipe_launches{0};

namespace {
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    cudaGetLastError();
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}
}  // namespace

// whether the pipelined pass can take this pass: the middle (y) pass in place
// over groups of N rows of pitch S, realizations back to back, 16-byte rows
static bool tma_pass_ok(const AxisArgs& a, int n, const void* in, const void* out) {
  return a.axis == 1 && in == out && a.gstride == (long long)n * a.S &&
         (a.nreal == 1 || a.rstride == (long long)a.ngroups * a.gstride) && (a.S * 8) % 16 == 0 &&
         ((uintptr_t)out % 16) == 0 && (long long)a.ngroups * a.nreal < (1LL << 31) && encode_tiled() != nullptr;
}

template <int L, int P>
static cudaError_t run_axis_c2c_tma(const AxisArgs& a, const Geo& g, float2* out, Tw tw, cudaStream_t st) {
  using LY = TmaLayout<L, P>;
  CUtensorMap map;
  const cuuint64_t dims[3] = {(cuuint64_t)a.S, (cuuint64_t)LY::N, (cuuint64_t)a.ngroups * (cuuint64_t)a.nreal};
  const cuuint64_t strides[2] = {(cuuint64_t)a.S * 8, (cuuint64_t)a.gstride * 8};
  const cuuint32_t box[3] = {(cuuint32_t)LY::LPT, (cuuint32_t)LY::ROWS, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  // complex FP32 values move as 8-byte elements; columns past the row pitch read as zeros
  if (encode_tiled()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, out, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  auto kern = k_col_tma<L, P>;
  cudaError_t e = func_smem(reinterpret_cast<const void*>(kern), LY::SMEM);
  if (e != cudaSuccess) return e;
  static int occ[2][16] = {};   // resident CTAs per SM, per variant and length (same on every B200)
  int& o = occ[P][L];
  if (o == 0) {
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, LY::NTH, LY::SMEM);
    if (e != cudaSuccess) return e;
    o = std::max(o, 1);
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  AxisArgs b = a;
  b.tpg = (a.lines + LY::LPT - 1) / LY::LPT;
  const long long ntiles = (long long)b.tpg * a.ngroups * a.nreal;
  if (ntiles <= 0) return cudaSuccess;
  if (ntiles >= (1LL << 31)) return cudaErrorInvalidValue;
  const int grid = (int)std::min<long long>(ntiles, (long long)nsm * o);
  kern<<<grid, LY::NTH, LY::SMEM, st>>>(b, g, out, tw, map, (int)ntiles);
  ++g_launch_count;
  ++g_pipe_launches;
  return cudaGetLastError();
}

// Reads and clears the flag a timed-out copy wait leaves behind; true if set.
bool pipe_error_take(cudaStream_t st) {
  int v = 0;
  if (cudaMemcpyFromSymbolAsync(&v, g_pipe_err, sizeof v, 0, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  if (v) {
    const int zero = 0;
    cudaMemcpyToSymbolAsync(g_pipe_err, &zero, sizeof zero, 0, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
  }
  return v != 0;
}

template <typename R, int L, int V>
static cudaError_t run_axis_gen_v(const AxisArgs& a, const Geo& g, const R* amp, const uint32_t* rs,
                                  const uint32_t* apow, cpx_t<R>* out, Tw tw, cudaStream_t st) {
  using CF = AxisCfg<R, L, V>;
  if constexpr (L == 0) {
    return cudaErrorInvalidValue;
  } else {
    size_t smem = (size_t)(CF::N * CF::TX + CF::N) * CF::EB;
    auto kern = g.d == 2 ? k_colgen<R, L, V, 1> : k_colgen<R, L, V, 0>;
    // pruned forms as in run_axis_c2c_v
    if constexpr (half_len(L) && (V < 4 || L >= 7))
      if (2 * a.nout <= CF::N) kern = g.d == 2 ? k_colgen<R, L, V, 1, true> : k_colgen<R, L, V, 0, true>;
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    AxisArgs b = a;
    b.tpg = (a.lines + CF::LPT - 1) / CF::LPT;
    unsigned blocks = (unsigned)((long long)b.tpg * a.ngroups * a.nreal);
    kern<<<blocks, CF::NTH, smem, st>>>(b, g, amp, rs, apow, out, tw);
    ++g_launch_count;
    return cudaGetLastError();
  }
}

template <typename R, typename O, int L, int V>
static cudaError_t run_rows_c2r_v(const Geo& g, const cpx_t<R>* in, long long rstride, O* out, long long ostride,
                                  int nreal, double* part, int* nblk_out, Tw tw, cudaStream_t st) {
  using RC = RowCfg<R, L, V>;
  constexpr int N = RC::N;
  size_t smem = (size_t)((N + 1) * RC::PITCH + 3 * N) * sizeof(cpx_t<R>);
  cudaError_t e = set_smem(k_rows_c2r<R, O, L, V>, smem);
  if (e != cudaSuccess) return e;
  int nblk = (g.ny * g.nz + RC::TX - 1) / RC::TX;
  if (nblk_out) *nblk_out = nblk;
  k_rows_c2r<R, O, L, V><<<(unsigned)((long long)nblk * nreal), RC::NTH, smem, st>>>(g, in, rstride, out, ostride,
                                                                                     nreal, nblk, part, tw);
  ++g_launch_count;
  return cudaGetLastError();
}

// row pass variant 4: rows held in warps, for the lengths RowWarpCfg covers
template <typename R, typename O, int L>
static cudaError_t run_rows_warp(const Geo& g, const cpx_t<R>* in, long long rstride, O* out, long long ostride,
                                 int nreal, double* part, int* nblk_out, Tw tw, cudaStream_t st) {
  using W = RowWarpCfg<R, L>;
  if constexpr (!W::ok) {
    return run_rows_c2r_v<R, O, L, 0>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
  } else {
    auto kern = k_rows_warp<R, O, L>;
    if constexpr (half_len(L))
      if ((g.nx + 1) / 2 <= W::N / 2) kern = k_rows_warp<R, O, L, true>;
    cudaError_t e = set_smem(kern, W::smem);
    if (e != cudaSuccess) return e;
    int nblk = (g.ny * g.nz + W::ROWS - 1) / W::ROWS;
    if (nblk_out) *nblk_out = nblk;
    kern<<<(unsigned)((long long)nblk * nreal), W::NTH, W::smem, st>>>(g, in, rstride, out, ostride, nreal, nblk,
                                                                       part, tw);
    ++g_launch_count;
    return cudaGetLastError();
  }
}

// row pass variant 6: two rows per lane on packed FP32, for the lengths
// RowPairCfg covers (variant 4 elsewhere, and for FP64)
template <typename R, typename O, int L>
static cudaError_t run_rows_pair(const Geo& g, const cpx_t<R>* in, long long rstride, O* out, long long ostride,
                                 int nreal, double* part, int* nblk_out, Tw tw, cudaStream_t st) {
  using W = RowPairCfg<L>;
  if constexpr (sizeof(R) != 4 || !W::ok) {
    return run_rows_warp<R, O, L>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
  } else {
    cudaError_t e = set_smem(k_rows_pair<O, L>, W::smem);
    if (e != cudaSuccess) return e;
    int nblk = (g.ny * g.nz + W::ROWS - 1) / W::ROWS;
    if (nblk_out) *nblk_out = nblk;
    k_rows_pair<O, L><<<(unsigned)((long long)nblk * nreal), W::NTH, W::smem, st>>>(
        g, reinterpret_cast<const float2*>(in), rstride, out, ostride, nreal, nblk, part, tw);
    ++g_launch_count;
    return cudaGetLastError();
  }
}

// variants are compiled for transform lengths 32..1024; other lengths use variant 0
constexpr bool tuned_len(int L) { return L >= 5 && L <= 10; }
template <typename R> constexpr int prec_index() { return sizeof(R) == 4 ? 1 : 0; }

template <typename R, int L, int SIGN>
static cudaError_t run_axis_c2c(const AxisArgs& a, const Geo& g, const cpx_t<R>* in, cpx_t<R>* out, Tw tw,
                                cudaStream_t st) {
  if constexpr (tuned_len(L)) {
    switch (g_variant[0][prec_index<R>()][L]) {
      case 1: return run_axis_c2c_v<R, L, SIGN, 1>(a, g, in, out, tw, st);
      case 2: return run_axis_c2c_v<R, L, SIGN, 2>(a, g, in, out, tw, st);
      case 3: return run_axis_c2c_v<R, L, SIGN, 3>(a, g, in, out, tw, st);
      default: break;
    }
    if constexpr (sizeof(R) == 4) {
      switch (g_variant[0][1][L]) {
        case 4: return run_axis_c2c_v<R, L, SIGN, 4>(a, g, in, out, tw, st);
        case 5: return run_axis_c2c_v<R, L, SIGN, 5>(a, g, in, out, tw, st);
        case 6: return run_axis_c2c_v<R, L, SIGN, 6>(a, g, in, out, tw, st);
        case 7: return run_axis_c2c_v<R, L, SIGN, 7>(a, g, in, out, tw, st);
        default: break;
      }
      // 8, 9: tiles staged by bulk tensor copies (inverse middle pass only;
      // other passes run the same tile shape with direct loads)
      const int v = g_variant[0][1][L];
      if (SIGN > 0 && (v == 8 || v == 9)) {
        if (tma_pass_ok(a, 1 << L, in, out)) {
          if (v == 8) return run_axis_c2c_tma<L, 0>(a, g, reinterpret_cast<float2*>(out), tw, st);
          return run_axis_c2c_tma<L, 1>(a, g, reinterpret_cast<float2*>(out), tw, st);
        }
        if (v == 8) return run_axis_c2c_v<R, L, SIGN, 0>(a, g, in, out, tw, st);
        return run_axis_c2c_v<R, L, SIGN, 4>(a, g, in, out, tw, st);
      }
    }
  }
  return run_axis_c2c_v<R, L, SIGN, 0>(a, g, in, out, tw, st);
}

template <typename R, int L>
static cudaError_t run_axis_gen(const AxisArgs& a, const Geo& g, const R* amp, const uint32_t* rs,
                                const uint32_t* apow, cpx_t<R>* out, Tw tw, cudaStream_t st) {
  if constexpr (tuned_len(L)) {
    switch (g_variant[1][prec_index<R>()][L]) {
      case 1: return run_axis_gen_v<R, L, 1>(a, g, amp, rs, apow, out, tw, st);
      case 2: return run_axis_gen_v<R, L, 2>(a, g, amp, rs, apow, out, tw, st);
      case 3: return run_axis_gen_v<R, L, 3>(a, g, amp, rs, apow, out, tw, st);
      default: break;
    }
    if constexpr (sizeof(R) == 4) {
      switch (g_variant[1][1][L]) {
        case 4: return run_axis_gen_v<R, L, 4>(a, g, amp, rs, apow, out, tw, st);
        case 5: return run_axis_gen_v<R, L, 5>(a, g, amp, rs, apow, out, tw, st);
        case 6: return run_axis_gen_v<R, L, 6>(a, g, amp, rs, apow, out, tw, st);
        case 7: return run_axis_gen_v<R, L, 7>(a, g, amp, rs, apow, out, tw, st);
        default: break;
      }
    }
  }
  return run_axis_gen_v<R, L, 0>(a, g, amp, rs, apow, out, tw, st);
}

template <typename R, typename O, int L>
static cudaError_t run_rows_c2r(const Geo& g, const cpx_t<R>* in, long long rstride, O* out, long long ostride,
                                int nreal, double* part, int* nblk_out, Tw tw, cudaStream_t st) {
  if constexpr (tuned_len(L)) {
    switch (g_variant[2][prec_index<R>()][L]) {
      case 1: return run_rows_c2r_v<R, O, L, 1>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
      case 2: return run_rows_c2r_v<R, O, L, 2>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
      case 3: return run_rows_c2r_v<R, O, L, 3>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
      case 4:   // 5 (the fused middle + row pass) where it does not apply runs variant 4
      case 5: return run_rows_warp<R, O, L>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
      case 6: return run_rows_pair<R, O, L>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
      default: break;
    }
  }
  return run_rows_c2r_v<R, O, L, 0>(g, in, rstride, out, ostride, nreal, part, nblk_out, tw, st);
}

template <int L>
static cudaError_t run_col_amp(const AxisArgs& a, const Geo& g, const double2* in, double* amp64, float* amp32, Tw tw,
                               SpecPartial* part, int npart_max, int* nb, cudaStream_t st) {
  if constexpr (L == 0) {
    return cudaErrorInvalidValue;
  } else {
    using CF = ColCfg<double, L, 0>;
    const size_t smem = (size_t)(CF::N * CF::TX + CF::N) * sizeof(double2);
    cudaError_t e = set_smem(k_col_amp<L>, smem);
    if (e != cudaSuccess) return e;
    const int blocks = (a.lines + CF::TX - 1) / CF::TX;
    if (blocks > npart_max) return cudaErrorInvalidValue;
    *nb = blocks;
    k_col_amp<L><<<blocks, CF::NTH, smem, st>>>(a, g, in, amp64, amp32, tw, part);
    ++g_launch_count;
    return cudaGetLastError();
  }
}

// partial-sum entries the spectrum build needs for grid g (one per block of
// the amplitude step), plus one for the result
int spectrum_parts(const Geo& g) {
  if (g.npz > 1) {
    const int L = ilog2(g.npz);
    const int tx = std::min(64, std::max(2, 4096 >> L));   // ColCfg<double, L, 0>::TX
    const long long lines = (long long)g.npy * g.HP;
    return (int)std::max<long long>(148 * 8, (lines + tx - 1) / tx) + 1;
  }
  return 148 * 8 + 1;
}

template <int L>
static cudaError_t run_spec_rows(const Model& m, const double d[3], const Geo& g, double2* out, Tw tw,
                                 cudaStream_t st) {
  constexpr int TX = RowTX<double, L>::TX;
  constexpr int N = 1 << L;
  if constexpr (SpecWarpCfg<L>::ok) {   // rows in warps
    using W = SpecWarpCfg<L>;
    cudaError_t e = set_smem(k_spec_rows_warp<L>, W::smem);
    if (e != cudaSuccess) return e;
    const int nblk = (g.npy * g.npz + W::ROWS - 1) / W::ROWS;
    k_spec_rows_warp<L><<<nblk, W::NTH, W::smem, st>>>(m, d[0], d[1], d[2], g, out, tw);
    ++g_launch_count;
    return cudaGetLastError();
  }
  size_t smem = (size_t)((N + 1) * (TX + 1) + 2 * N) * sizeof(double2) + (size_t)(TX + 1) * MAXST * 3 * sizeof(double);
  cudaError_t e = set_smem(k_spec_rows<L>, smem);
  if (e != cudaSuccess) return e;
  int nblk = (g.npy * g.npz + TX - 1) / TX;
  k_spec_rows<L><<<nblk, NT, smem, st>>>(m, d[0], d[1], d[2], g, out, tw);
  ++g_launch_count;
  return cudaGetLastError();
}

// fused middle + row passes (row variant 5): whether it takes grid g, and the launch
template <int LY, int LX, int CL>
static cudaError_t run_yx_cl(const Geo& g, const float2* work, long long wstride, int nreal, float* out, Tw tw,
                             cudaStream_t st) {
  using Y = YXCfg<LY, LX>;
  auto kern = k_yx_fused<LY, LX, CL>;
  cudaError_t e = func_smem(reinterpret_cast<const void*>(kern), Y::SMEM);
  if (e != cudaSuccess) return e;
  const long long blocks = (long long)g.nz * nreal * CL;
  if (blocks >= (1LL << 31)) return cudaErrorInvalidValue;
  kern<<<(unsigned)blocks, Y::NTH, Y::SMEM, st>>>(g, work, wstride, out, tw);
  ++g_launch_count;
  return cudaGetLastError();
}

template <int LY, int LX>
static cudaError_t run_yx(const Geo& g, const float2* work, long long wstride, int nreal, float* out, Tw tw,
                          cudaStream_t st) {
  using Y = YXCfg<LY, LX>;
  if constexpr (!Y::ok) {
    return cudaErrorInvalidValue;
  } else {
    const int need = (g.ny + Y::TXR - 1) / Y::TXR;   // CTAs that own rows
    if (need <= 2) return run_yx_cl<LY, LX, 2>(g, work, wstride, nreal, out, tw, st);
    if (need <= 4) return run_yx_cl<LY, LX, 4>(g, work, wstride, nreal, out, tw, st);
    return run_yx_cl<LY, LX, 8>(g, work, wstride, nreal, out, tw, st);
  }
}

static bool yx_fused_ok(const Geo& g) {
  const int Ly = ilog2(g.npy), Lx = ilog2(g.npx) - 1;
  if (g.npz < 2 || Ly < 6 || Ly > 9 || Lx < 7 || Lx > 9) return false;
  const int txr = std::min(64, std::max(1, 8192 >> Lx));   // RowCfg<float, Lx, 0>::TX
  return g.ny <= 8 * txr;
}

template <int LY>
static cudaError_t run_yx_lx(const Geo& g, const float2* work, long long wstride, int nreal, float* out, Tw tw,
                             cudaStream_t st) {
  switch (ilog2(g.npx) - 1) {
    case 7: return run_yx<LY, 7>(g, work, wstride, nreal, out, tw, st);
    case 8: return run_yx<LY, 8>(g, work, wstride, nreal, out, tw, st);
    case 9: return run_yx<LY, 9>(g, work, wstride, nreal, out, tw, st);
    default: return cudaErrorInvalidValue;
  }
}

static cudaError_t launch_yx_fused(const Geo& g, const float2* work, long long wstride, int nreal, float* out, Tw tw,
                                   cudaStream_t st) {
  switch (ilog2(g.npy)) {
    case 6: return run_yx_lx<6>(g, work, wstride, nreal, out, tw, st);
    case 7: return run_yx_lx<7>(g, work, wstride, nreal, out, tw, st);
    case 8: return run_yx_lx<8>(g, work, wstride, nreal, out, tw, st);
    case 9: return run_yx_lx<9>(g, work, wstride, nreal, out, tw, st);
    default: return cudaErrorInvalidValue;
  }
}

// x pass rows kernel: number of row blocks per realization (for the partial sums)
int realize_part_blocks(const Geo& g, bool dbl) {
  if (g.npx == 1) return (g.ny * g.nz + NT - 1) / NT;
  int L = ilog2(g.npx) - 1;
  int v = tuned_len(L) ? g_variant[2][dbl ? 0 : 1][L] : 0;
  // 5 (fused, never with statistics) and 6 outside its lengths run variant 4
  if (v == 5 || (v == 6 && (dbl || L < 3 || L > 8))) v = 4;
  if (v == 6) {   // RowPairCfg
    const int tpc = (1 << L) / 8;                       // lanes per row pair
    const int rows = 16 * (tpc >= 32 ? 1 : 32 / tpc);   // rows per block
    return (g.ny * g.nz + rows - 1) / rows;
  }
  if (v == 4 && L >= 3 && L <= (dbl ? 8 : 9)) {   // RowWarpCfg
    const int tpc = (1 << L) / (L > 8 ? 16 : 8);      // lanes per row
    const int rows = 8 * (tpc >= 32 ? 1 : 32 / tpc);  // rows per block
    return (g.ny * g.nz + rows - 1) / rows;
  }
  if (v >= 4) v = 0;   // 4 outside its lengths runs variant 0
  int E = (dbl ? 4096 : 8192) >> ((v >> 1) & 1);
  int tx = std::min(64, std::max(1, E >> L));
  return (g.ny * g.nz + tx - 1) / tx;
}

// ---------------------------------------------------------------- public launchers
cudaError_t launch_spectrum(const Model& m, const double d[3], const Geo& g, double2* work, double* amp64,
                            float* amp32, SpecPartial* part, int npart_max, SpecPartial* result, Tw tw,
                            cudaStream_t st) {
  cudaError_t e;
  if (g.npx == 1) {
    int nrows = g.npy * g.npz;
    k_spec_rows_n1<<<(nrows + NT - 1) / NT, NT, 0, st>>>(m, d[0], d[1], d[2], g, work);
    ++g_launch_count;
    e = cudaGetLastError();
  } else {
    int L = ilog2(g.npx) - 1;
    e = cudaErrorInvalidValue;
    SS3D_LOGN_SWITCH(L, MAX_LOGN_D, e = run_spec_rows<L>(m, d, g, work, tw, st));
  }
  if (e != cudaSuccess) return e;
  if (g.npy > 1) {
    AxisArgs a{};
    a.S = g.HP;
    a.nout = g.npy;
    a.lines = g.H;
    a.ngroups = g.npz;
    a.gstride = (long long)g.npy * g.HP;
    a.rstride = 0;
    a.nreal = 1;
    a.axis = 1;
    int L = ilog2(g.npy);
    e = cudaErrorInvalidValue;
    SS3D_LOGN_SWITCH(L, MAX_LOGN_D, e = (run_axis_c2c<double, L, -1>(a, g, work, work, tw, st)));
    if (e != cudaSuccess) return e;
  }
  int nb = 0;
  if (g.npz > 1) {
    // z pass with the amplitude step in its stores
    AxisArgs a{};
    a.S = (long long)g.npy * g.HP;
    a.nout = g.npz;
    a.lines = g.npy * g.HP;
    a.ngroups = 1;
    a.axis = 2;
    int L = ilog2(g.npz);
    e = cudaErrorInvalidValue;
    SS3D_LOGN_SWITCH(L, MAX_LOGN_D, e = (run_col_amp<L>(a, g, work, amp64, amp32, tw, part, npart_max, &nb, st)));
    if (e != cudaSuccess) return e;
  } else {
    long long tot = (long long)g.npz * g.npy * g.HP;
    nb = (int)std::min<long long>(npart_max, (tot + NT - 1) / NT);
    k_spec_amp<<<nb, NT, 0, st>>>(g, work, amp64, amp32, part);
    ++g_launch_count;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  k_reduce_spec<<<1, RS_NT, 0, st>>>(part, nb, result);
  ++g_launch_count;
  return cudaGetLastError();
}

template <int L, int SIGN>
static cudaError_t run_rows_c2c(long long nrows, double2* a, Tw tw, cudaStream_t st) {
  if constexpr (L == 0) {
    return cudaSuccess;   // length-1 rows: identity
  } else {
    constexpr int TX = RowTX<double, L>::TX;
    constexpr int N = 1 << L;
    const size_t smem = (size_t)(N * (TX + 1) + N) * sizeof(double2);
    cudaError_t e = set_smem(k_rows_c2c<L, SIGN>, smem);
    if (e != cudaSuccess) return e;
    const long long nblk = (nrows + TX - 1) / TX;
    if (nblk > 0x7fffffffLL) return cudaErrorInvalidValue;
    k_rows_c2c<L, SIGN><<<(unsigned)nblk, NT, smem, st>>>(nrows, a, tw);
    ++g_launch_count;
    return cudaGetLastError();
  }
}

// Unscaled 3D c2c transform of a full complex grid a[nz][ny][nx] in place
// (fft3d, f90:254-304): isign -1 forward (e^{-i}), +1 inverse; every axis a
// power of two up to 2^MAX_LOGN_D.
cudaError_t launch_fft3d(double2* a, int nx, int ny, int nz, int isign, Tw tw, cudaStream_t st) {
  const int Lx = ilog2(nx), Ly = ilog2(ny), Lz = ilog2(nz);
  if ((1 << Lx) != nx || (1 << Ly) != ny || (1 << Lz) != nz) return cudaErrorInvalidValue;
  Geo g{};
  g.npx = g.nx = nx;
  g.npy = g.ny = ny;
  g.npz = g.nz = nz;
  g.H = g.HP = nx;   // full rows: every line of a plane is valid
  cudaError_t e = cudaErrorInvalidValue;
  const long long rows = (long long)ny * nz;
  if (isign < 0) {
    SS3D_LOGN_SWITCH(Lx, MAX_LOGN_D, e = (run_rows_c2c<L, -1>(rows, a, tw, st)));
  } else {
    SS3D_LOGN_SWITCH(Lx, MAX_LOGN_D, e = (run_rows_c2c<L, +1>(rows, a, tw, st)));
  }
  if (e != cudaSuccess) return e;
  if (ny > 1) {
    AxisArgs b{};
    b.S = nx;
    b.nout = ny;
    b.lines = nx;
    b.ngroups = nz;
    b.gstride = (long long)nx * ny;
    b.rstride = 0;
    b.nreal = 1;
    b.axis = 1;
    e = cudaErrorInvalidValue;
    if (isign < 0) {
      SS3D_LOGN_SWITCH(Ly, MAX_LOGN_D, e = (run_axis_c2c<double, L, -1>(b, g, a, a, tw, st)));
    } else {
      SS3D_LOGN_SWITCH(Ly, MAX_LOGN_D, e = (run_axis_c2c<double, L, +1>(b, g, a, a, tw, st)));
    }
    if (e != cudaSuccess) return e;
  }
  if (nz > 1) {
    AxisArgs c{};
    c.S = (long long)nx * ny;
    c.nout = nz;
    c.lines = nx * ny;
    c.ngroups = 1;
    c.gstride = 0;
    c.rstride = 0;
    c.nreal = 1;
    c.axis = 2;
    e = cudaErrorInvalidValue;
    if (isign < 0) {
      SS3D_LOGN_SWITCH(Lz, MAX_LOGN_D, e = (run_axis_c2c<double, L, -1>(c, g, a, a, tw, st)));
    } else {
      SS3D_LOGN_SWITCH(Lz, MAX_LOGN_D, e = (run_axis_c2c<double, L, +1>(c, g, a, a, tw, st)));
    }
  }
  return e;
}

cudaError_t launch_rowstates(const Geo& g, uint32_t s0, long long r_first, int nreal, const uint32_t* ptab,
                             uint32_t* rowstates, uint32_t* apow, cudaStream_t st) {
  long long tot = (long long)g.npy * g.npz * nreal;
  int nb = (int)std::min<long long>(4096, (tot + NT - 1) / NT);
  k_rowstates<<<nb, NT, 0, st>>>(g, s0, r_first, nreal, ptab, rowstates);
  ++g_launch_count;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || apow == nullptr) return e;
  k_apow<<<(g.npx + NT - 1) / NT, NT, 0, st>>>(g.npx, g.d, ptab, apow);
  ++g_launch_count;
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_gen(const Geo& g, const R* amp, const uint32_t* rowstates, const uint32_t* apow,
                       cpx_t<R>* work, long long wstride, int nreal, cudaStream_t st) {
  long long tot = (long long)g.npz * g.npy * g.HP * nreal;
  int nb = (int)std::min<long long>(148 * 16, (tot + NT - 1) / NT);
  k_gen<R><<<nb, NT, 0, st>>>(g, amp, rowstates, apow, work, wstride, nreal);
  ++g_launch_count;
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_realize(const Geo& g, const R* amp, const uint32_t* rowstates, const uint32_t* apow,
                           cpx_t<R>* work, long long wstride, int nreal, void* out, int out_kind, double* part,
                           int* nblk_per_r, Tw tw, bool fused, cudaStream_t st, Marks* marks,
                           cudaEvent_t first_done) {
  constexpr int ML = MaxL<R>::v;
  cudaError_t e = cudaSuccess;
  mark(marks, 1, st);
  auto first_pass_done = [&]() { return first_done ? cudaEventRecord(first_done, st) : cudaSuccess; };
  // first inverse axis: z if present, else y, else only x
  if (g.npz > 1) {
    AxisArgs a{};
    a.S = (long long)g.npy * g.HP;
    a.nout = g.nz;
    a.lines = g.npy * g.HP;
    a.ngroups = 1;
    a.gstride = 0;
    a.rstride = wstride;
    a.nreal = nreal;
    a.axis = 2;
    int L = ilog2(g.npz);
    if (fused) {
      e = cudaErrorInvalidValue;
      SS3D_LOGN_SWITCH(L, ML, e = (run_axis_gen<R, L>(a, g, amp, rowstates, apow, work, tw, st)));
    } else {
      e = launch_gen<R>(g, amp, rowstates, apow, work, wstride, nreal, st);
      if (e != cudaSuccess) return e;
      e = cudaErrorInvalidValue;
      SS3D_LOGN_SWITCH(L, ML, e = (run_axis_c2c<R, L, +1>(a, g, work, work, tw, st)));
    }
    if (e == cudaSuccess) e = first_pass_done();
    if (e != cudaSuccess) return e;
    if (g.npy > 1) {
      if constexpr (sizeof(R) == 4) {
        // row variant 5: middle and row passes in one cluster kernel per plane
        const int Lx = ilog2(g.npx) - 1;
        if (out_kind == 0 && part == nullptr && Lx >= 0 && Lx < 16 && g_variant[2][1][Lx] == 5 &&
            yx_fused_ok(g)) {
          mark(marks, 3, st);
          return launch_yx_fused(g, work, wstride, nreal, (float*)out, tw, st);
        }
      }
      mark(marks, 2, st);
      AxisArgs b{};
      b.S = g.HP;
      b.nout = g.ny;
      b.lines = g.H;
      b.ngroups = g.nz;
      b.gstride = (long long)g.npy * g.HP;
      b.rstride = wstride;
      b.nreal = nreal;
      b.axis = 1;
      int Ly = ilog2(g.npy);
      e = cudaErrorInvalidValue;
      SS3D_LOGN_SWITCH(Ly, ML, e = (run_axis_c2c<R, L, +1>(b, g, work, work, tw, st)));
      if (e != cudaSuccess) return e;
    }
  } else if (g.npy > 1) {
    AxisArgs b{};
    b.S = g.HP;
    b.nout = g.ny;
    b.lines = g.H;
    b.ngroups = 1;
    b.gstride = (long long)g.npy * g.HP;
    b.rstride = wstride;
    b.nreal = nreal;
    b.axis = 1;
    int Ly = ilog2(g.npy);
    if (fused) {
      e = cudaErrorInvalidValue;
      SS3D_LOGN_SWITCH(Ly, ML, e = (run_axis_gen<R, L>(b, g, amp, rowstates, apow, work, tw, st)));
    } else {
      e = launch_gen<R>(g, amp, rowstates, apow, work, wstride, nreal, st);
      if (e != cudaSuccess) return e;
      e = cudaErrorInvalidValue;
      SS3D_LOGN_SWITCH(Ly, ML, e = (run_axis_c2c<R, L, +1>(b, g, work, work, tw, st)));
    }
    if (e == cudaSuccess) e = first_pass_done();
    if (e != cudaSuccess) return e;
  } else {
    e = launch_gen<R>(g, amp, rowstates, apow, work, wstride, nreal, st);
    if (e == cudaSuccess) e = first_pass_done();
    if (e != cudaSuccess) return e;
  }
  // x pass
  mark(marks, 3, st);
  const long long ostride = (long long)g.nx * g.ny * g.nz;
  if (g.npx == 1) {
    int nblk = (g.ny * g.nz + NT - 1) / NT;
    if (nblk_per_r) *nblk_per_r = nblk;
    if (out_kind == 0)
      k_rows_copy<R, float><<<nblk * nreal, NT, 0, st>>>(g, work, wstride, (float*)out, ostride, nreal, nblk, part);
    else
      k_rows_copy<R, double><<<nblk * nreal, NT, 0, st>>>(g, work, wstride, (double*)out, ostride, nreal, nblk,
                                                          part);
    ++g_launch_count;
    return cudaGetLastError();
  }
  int Lx = ilog2(g.npx) - 1;
  e = cudaErrorInvalidValue;
  if (out_kind == 0) {
    SS3D_LOGN_SWITCH(Lx, ML,
                     e = (run_rows_c2r<R, float, L>(g, work, wstride, (float*)out, ostride, nreal, part,
                                                     nblk_per_r, tw, st)));
  } else {
    SS3D_LOGN_SWITCH(Lx, ML,
                     e = (run_rows_c2r<R, double, L>(g, work, wstride, (double*)out, ostride, nreal, part,
                                                      nblk_per_r, tw, st)));
  }
  return e;
}

cudaError_t launch_debug_states(const Geo& g, const uint32_t* rowstates, const uint32_t* apow, uint32_t* out,
                                cudaStream_t st) {
  long long tot = (long long)g.npz * g.npy * g.H;
  int nb = (int)std::min<long long>(4096, (tot + NT - 1) / NT);
  k_debug_states<<<nb, NT, 0, st>>>(g, rowstates, apow, out);
  ++g_launch_count;
  return cudaGetLastError();
}

cudaError_t launch_reduce_zstats(const double* part, int nblk_per_r, int nreal, double* zsum, cudaStream_t st) {
  k_reduce_zstats<<<nreal, NT, 0, st>>>(part, nblk_per_r, zsum);
  ++g_launch_count;
  return cudaGetLastError();
}

template cudaError_t launch_realize<float>(const Geo&, const float*, const uint32_t*, const uint32_t*, float2*,
                                           long long, int, void*, int, double*, int*, Tw, bool, cudaStream_t,
                                           Marks*, cudaEvent_t);
template cudaError_t launch_realize<double>(const Geo&, const double*, const uint32_t*, const uint32_t*, double2*,
                                            long long, int, void*, int, double*, int*, Tw, bool, cudaStream_t,
                                            Marks*, cudaEvent_t);
template cudaError_t launch_gen<float>(const Geo&, const float*, const uint32_t*, const uint32_t*, float2*,
                                       long long, int, cudaStream_t);
template cudaError_t launch_gen<double>(const Geo&, const double*, const uint32_t*, const uint32_t*, double2*,
                                        long long, int, cudaStream_t);

const void* module_anchor_fft() { return reinterpret_cast<const void*>(k_rowstates); }

}  // namespace ss3d
