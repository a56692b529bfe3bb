// ss3d_bodies.cuh -- bodies of the three realization passes as device
// functions of a work-item index, shared by the per-pass kernels (one CTA per
// item, ss3d_fft.cu) and the batch kernels (CTAs over the items of many grids,
// ss3d_batch.cu).
//
//   colgen_body  synthesis of the Hermitian coefficients (reference fill
//                f90:1305-1334) fused with the first inverse axis pass
//   col_body     inverse pass along a strided axis, pruned to the crop
//   rows_body    C2R pass along x with the crop (f90:1335-1340)
#pragma once
#include "ss3d_engine.cuh"
#include "ss3d_internal.h"

namespace ss3d {

template <typename R> __device__ __forceinline__ const cpx_t<R>* twtab(const Tw& tw);
template <> __device__ __forceinline__ const float2* twtab<float>(const Tw& tw) { return tw.f; }
template <> __device__ __forceinline__ const double2* twtab<double>(const Tw& tw) { return tw.d; }

// ---------------------------------------------------------------- strided axis passes
// A "line" is one column along the transformed axis.  Lines of one group are
// contiguous in memory; groups are gstride apart; realizations rstride apart.
struct AxisArgs {
  long long S;         // element stride along the axis
  int nout;            // positions stored (p < nout)
  int lines;           // lines per group
  int ngroups;
  long long gstride;
  int tpg;             // tiles per group
  long long rstride;   // realization stride in the complex buffer
  int nreal;
  int axis;            // 1 = y, 2 = z (index decoding of the synthesis)
};

__device__ __forceinline__ bool line_valid(const Geo& g, int line, int lines) {
  return line < lines && (line % g.HP) < g.H;
}

// ---------------------------------------------------------------- register-resident column passes
// Tile configuration per transform length: TX columns, TPC threads per column,
// ET = N / TPC elements per thread (16 in float, 8 in double).
// Variant V (tuned at run time): bit 0 halves the elements per thread
// (more threads, fewer registers), bit 1 halves the tile (fewer columns).
template <typename R, int LOGN, int V = 0> struct ColCfg {
  static constexpr int N = 1 << LOGN;
  static constexpr int ETW0 = sizeof(R) == 4 ? 16 : 8;
  static constexpr int ETW = (V & 1) ? (ETW0 / 2 < 8 ? 8 : ETW0 / 2) : ETW0;
  static constexpr int ET = N < ETW ? N : ETW;
  static constexpr int TPC = N / ET;
  static constexpr int E = (sizeof(R) == 4 ? 8192 : 4096) >> ((V >> 1) & 1);
  static constexpr int TX0 = E / N;
  static constexpr int TX = TX0 > 64 ? 64 : (TX0 < 2 ? 2 : TX0);
  static constexpr int NTH = TX * TPC;
  static_assert(NTH <= 1024, "tile too large");
};

// c2c transform along a strided axis (in place allowed), unscaled, pruned store
template <typename R, int LOGN, int TX, int TPC, int SIGN, bool HALF = false>
__device__ __forceinline__ void col_body(const AxisArgs& a, const Geo& g, const cpx_t<R>* in, cpx_t<R>* out,
                                         const Tw& tw, int item, unsigned char* smraw) {
  using C = cpx_t<R>;
  constexpr int N = 1 << LOGN;
  constexpr int NTH = TX * TPC;
  C* s = reinterpret_cast<C*>(smraw);
  C* stw = s + N * TX;
  const int r = item % a.nreal;
  const int tile = item / a.nreal;
  const int grp = tile / a.tpg;
  const int line0 = (tile % a.tpg) * TX;
  const int t = threadIdx.x % TX;
  const bool valid = line_valid(g, line0 + t, a.lines);
  // a line past the grid reads line 0 (in range) and stores nothing: the
  // columns of a tile are independent transforms, so no select in the loader
  const C* src = in + ((long long)grp * a.gstride + (valid ? line0 + t : 0) + (long long)r * a.rstride);
  C* dst = out + ((long long)grp * a.gstride + line0 + t + (long long)r * a.rstride);
  const int S = (int)a.S;   // offsets inside one realization's grid fit in 32 bits
  const int nout = a.nout;
  constexpr int NR0 = N / Sched<LOGN>::radix(0);
  for (int q = threadIdx.x; q < N; q += NTH) stw[q] = twtab<R>(tw)[N - 1 + q];
  __syncthreads();
  fft_tile<LOGN, TX, TPC, SIGN, TX, false, false, HALF>(
      s, stw, [&](int jb, int r) { return src[(jb + r * NR0) * S]; },
      [&](int pos, C v) {
        if (valid && pos < nout) dst[pos * S] = v;
      });
}

// Coefficient from the Park-Miller state s1 of its first draw (f90:1312-1331):
// GAUSS 1: amp (g1 + i g2) sqrt(1/2) from the Box-Muller pair of draws s1, s1 a;
// GAUSS 0: amp e^{i phi}, phi = 2 pi u(s1).  A self-conjugate index takes
// amp g1 (Gaussian) or +/-amp (phases: + when u < 1/2); conj gives the
// conjugate (index whose draw belongs to its partner).  Branch-free.
template <typename R, int GAUSS>
__device__ __forceinline__ cpx_t<R> coef_from_state(uint32_t s1, R am, bool self, bool conj) {
  using C = cpx_t<R>;
  if constexpr (GAUSS) {
    const uint32_t s2 = sizeof(R) == 4 ? pm_mulmod_lazy(s1, PM_A) : pm_mulmod(s1, PM_A);
    if constexpr (sizeof(R) == 4) {
      const float L = m2log_f(s1);
      const float rr = L * rsqrt_hw(L);
      float cs, sn;
      const bool odd = phasor_half_f(s2, cs, sn);
      const float t0 = (self ? am : am * 0.70710678118654752f) * rr;
      const float t = odd ? -t0 : t0;
      const float re = t * cs;
      const float im = (conj ? -t : t) * sn;
      return cmk<C>(re, self ? 0.f : im);
    } else {
      const double rr = sqrt(m2log_d(s1));
      double cs, sn;
      phasor_d(s2, cs, sn);
      const double g1 = rr * cs, g2 = rr * sn;
      const double h = 0.70710678118654757;   // sqrt(0.5d0)
      const double re = self ? am * g1 : am * g1 * h;
      const double im = am * (conj ? -g2 : g2) * h;
      return cmk<C>(re, self ? 0.0 : im);
    }
  } else {
    R cs, sn, a = am;
    if constexpr (sizeof(R) == 4) {
      if (phasor_half_f(s1, cs, sn)) a = -a;
    } else {
      phasor_d(s1, cs, sn);
    }
    const R sgn = (2ull * s1) < (uint64_t)PM_M ? am : -am;   // urand() < 0.5
    const R re = self ? sgn : a * cs;
    const R im = conj ? -(a * sn) : a * sn;
    return cmk<C>(re, self ? R(0) : im);
  }
}

// The coefficients of the two lanes of a pair (states s0, s1 of their first
// draws, amplitudes am): the operations of coef_from_state<float, GAUSS> lane
// by lane, with the products and the logarithm's series on packed FP32
// instructions and the hardware functions and integer steps per lane.
__device__ __forceinline__ float2 m2log_f2(uint32_t s0, uint32_t s1) {
  const float2 a = make_float2((float)(PM_M - s0), (float)(PM_M - s1));
  const float2 b = ksub(kconst<float2>(4294967294.0), a);
  const float2 q = kmul(a, make_float2(rcp_hw(b.x), rcp_hw(b.y)));
  const float2 z2 = kmul(q, q);
  float2 p = kfma(z2, kconst<float2>(4.0f / 7.0f), kconst<float2>(4.0f / 5.0f));
  p = kfma(z2, p, kconst<float2>(4.0f / 3.0f));
  p = kfma(z2, p, kconst<float2>(4.0));
  const float2 near1 = kmul(p, q);
  const float2 far = kfma(kconst<float2>(-1.3862944f), make_float2(lg2_hw((float)s0), lg2_hw((float)s1)),
                          kconst<float2>(M2LOG_C31));
  return make_float2(s0 >= 1610612736u ? near1.x : far.x, s1 >= 1610612736u ? near1.y : far.y);
}
// cos and sin of the two remainders; sb0/sb1 hold the sign of the phasor in
// bit 31 (set for an odd half-turn count, as phasor_half_f's result), for
// callers that apply it to a factor by flipping that bit
__device__ __forceinline__ void phasor_half_f2(uint32_t s0, uint32_t s1, float2& c, float2& sn, uint32_t& sb0,
                                               uint32_t& sb1) {
  const int n0 = half_turns(s0), n1 = half_turns(s1);
  const float2 x = kmul(make_float2((float)half_turn_rem(s0, n0), (float)half_turn_rem(s1, n1)),
                        kconst<float2>(1.4629181e-9f));
  sn = make_float2(sin_hw(x.x), sin_hw(x.y));
  c = make_float2(cos_hw(x.x), cos_hw(x.y));
  sb0 = (uint32_t)n0 << 31;
  sb1 = (uint32_t)n1 << 31;
}
// v with its sign bit flipped where sb has bit 31 set (exactly -v then)
__device__ __forceinline__ float sign_flip(float v, uint32_t sb) { return __uint_as_float(__float_as_uint(v) ^ sb); }
template <int GAUSS>
__device__ __forceinline__ cpair coef_pair(uint32_t s0, uint32_t s1, float2 am, bool self0, bool self1, bool conj) {
  if constexpr (GAUSS) {
    const float2 L = m2log_f2(s0, s1);
    const float2 rr = kmul(L, make_float2(rsqrt_hw(L.x), rsqrt_hw(L.y)));
    float2 cs, sn;
    uint32_t sb0, sb1;
    phasor_half_f2(pm_mulmod_lazy(s0, PM_A), pm_mulmod_lazy(s1, PM_A), cs, sn, sb0, sb1);
    const float2 ah = kmul(am, kconst<float2>(0.70710678118654752f));
    const float2 t0 = kmul(make_float2(self0 ? am.x : ah.x, self1 ? am.y : ah.y), rr);
    const float2 t = make_float2(sign_flip(t0.x, sb0), sign_flip(t0.y, sb1));
    const float2 re = kmul(t, cs);
    const float2 im = kmul(conj ? kneg(t) : t, sn);
    return cpair{re, make_float2(self0 ? 0.f : im.x, self1 ? 0.f : im.y)};
  } else {
    float2 cs, sn;
    uint32_t sb0, sb1;
    phasor_half_f2(s0, s1, cs, sn, sb0, sb1);
    const float2 a = make_float2(sign_flip(am.x, sb0), sign_flip(am.y, sb1));
    const float2 re = kmul(a, cs);
    const float2 im0 = kmul(a, sn);
    const float2 im = conj ? kneg(im0) : im0;
    const float sg0 = (2ull * s0) < (uint64_t)PM_M ? am.x : -am.x, sg1 = (2ull * s1) < (uint64_t)PM_M ? am.y : -am.y;
    return cpair{make_float2(self0 ? sg0 : re.x, self1 ? sg1 : re.y),
                 make_float2(self0 ? 0.f : im.x, self1 ? 0.f : im.y)};
  }
}

// Row state that the draw of position p takes (rs_own: its own rows, rs_par:
// the partner rows).  Row states are [j][k] with k fastest, so consecutive
// positions along z hold consecutive states; along y (the first pass of a 2D
// grid) npz = 1 makes them consecutive too.  The partner position (N - p) mod N
// is N - p in the slots r >= 1 of pass 0 (p >= N/R0 > 0); in slot 0 only p = 0
// takes the partner's draw, whose partner position is 0.  r is a compile-time
// constant in the loaders, so every address is a per-thread base plus an
// immediate offset.
__device__ __forceinline__ const uint32_t* partner_state(const uint32_t* rs_own, const uint32_t* rs_par, int p,
                                                         int r, bool greater, int N) {
  return greater ? (r == 0 ? rs_par : rs_par + (N - p)) : rs_own + p;
}

// First inverse pass with the coefficient synthesis fused into the loader.
// axis 2: columns are (i, j) plane offsets, positions k;  axis 1 (npz = 1):
// columns are i, positions j.  Along the transformed axis (length N) the
// position p and its conjugate partner pp = (N - p) mod N decide which draw a
// coefficient takes: p < N/2 its own row's (less), p > N/2 the partner row's
// (conjugated), and p in {0, N/2} (partner = itself) the other index decides,
// as the reference's lin/linp comparison (f90:1315-1331) does.  The pass-0
// loader sees p = jb + r N/R0 with r constant, so only the two slots r = 0 and
// r = R0/2 of the butterflies with jb = 0 need a run-time decision.
template <typename R, int LOGN, int TX, int TPC, int GAUSS, bool HALF = false>
__device__ __forceinline__ void colgen_body(const AxisArgs& a, const Geo& g, const R* __restrict__ amp,
                                            const uint32_t* __restrict__ rowstates,
                                            const uint32_t* __restrict__ apow, cpx_t<R>* out, const Tw& tw,
                                            int item, unsigned char* smraw) {
  using C = cpx_t<R>;
  constexpr int N = 1 << LOGN;
  constexpr int NTH = TX * TPC;
  constexpr int R0 = Sched<LOGN>::radix(0);
  constexpr int NR0 = N / R0;
  C* s = reinterpret_cast<C*>(smraw);
  C* stw = s + N * TX;
  const int r = item % a.nreal;
  const int tile = item / a.nreal;
  const int grp = tile / a.tpg;
  const int line0 = (tile % a.tpg) * TX;
  const int t = threadIdx.x % TX;
  const int line = line0 + t;
  const bool valid = line_valid(g, line, a.lines);
  // lines past the grid or in the row padding compute with line 0's indices
  // (in range) and store nothing: no branch or select in the loader
  const int lsafe = valid ? line : 0;
  const bool zaxis = a.axis == 2;
  const int i = zaxis ? lsafe % g.HP : lsafe;
  const int j0 = zaxis ? lsafe / g.HP : 0;
  const uint32_t ai = __ldg(apow + i), aip = __ldg(apow + ((g.npx - i) & (g.npx - 1)));
  const bool iedge = (i == 0) || (2 * i == g.npx);
  // z pass: rows (j0, p) and (jp0, pp); y pass (2D): rows p and pp of plane 0
  const int jp0 = (-j0) & (g.npy - 1);
  const bool cgt = zaxis && j0 > jp0;                      // mid positions: partner's draw
  const bool selfcol = (!zaxis || j0 == jp0) && iedge;     // mid positions: self-conjugate
  const uint32_t* rs = rowstates + (size_t)r * g.npy * g.npz;
  const uint32_t* rs_own = rs + (zaxis ? (size_t)j0 * g.npz : 0);
  const uint32_t* rs_par = rs + (zaxis ? (size_t)jp0 * g.npz : 0);
  const long long cbase = (long long)grp * a.gstride + lsafe;
  const R* ap = amp + cbase;
  C* dst = out + cbase + (long long)r * a.rstride;
  const int S = (int)a.S;   // offsets inside one realization's grid fit in 32 bits
  const int nout = a.nout;
  for (int q = threadIdx.x; q < N; q += NTH) stw[q] = twtab<R>(tw)[N - 1 + q];
  __syncthreads();
  fft_tile<LOGN, TX, TPC, +1, TX, false, false, HALF>(
      s, stw,
      [&](int jb, int rr) {
        const int p = jb + rr * NR0;
        const R am = __ldg(ap + p * S);
        bool greater, mid;
        if (rr == 0) {                 // p < N/R0 <= N/2; p = 0 when jb = 0
          mid = jb == 0;
          greater = mid && cgt;
        } else if (2 * rr == R0) {     // p >= N/2; p = N/2 when jb = 0
          mid = jb == 0;
          greater = !mid || cgt;
        } else {
          mid = false;
          greater = 2 * rr > R0;
        }
        const uint32_t st = __ldg(partner_state(rs_own, rs_par, p, rr, greater, N));
        const uint32_t s1 = pm_mulmod(st, greater ? aip : ai);
        return coef_from_state<R, GAUSS>(s1, am, mid && selfcol, greater);
      },
      [&](int pos, C v) {
        if (valid && pos < nout) dst[pos * S] = v;
      });
}

// ---------------------------------------------------------------- column-pair passes (FP32)
// The same two passes with two adjacent lines per thread held as a cpair (real
// parts of both in x, imaginary parts in y): every butterfly operation is one
// packed sm_100 instruction for two elements, and the two complex values are
// one 16-byte access.  Lines 2u and 2u+1 lie in the same row (the row pitch HP
// is even).  The operations per lane are those of the one-line bodies, so the
// results are the same bits.  Variant bit 1 halves the tile, bit 0 doubles
// the pairs per thread.
template <int LOGN, int V = 0> struct PairCfg {
  static constexpr int N = 1 << LOGN;
  static constexpr int ETW = (V & 1) ? 16 : 8;
  static constexpr int ET = N < ETW ? N : ETW;    // pairs per thread
  static constexpr int TPC = N / ET;
  static constexpr int E = 4096 >> ((V >> 1) & 1);
  static constexpr int TX0 = E / N;
  static constexpr int TX = TX0 > 64 ? 64 : (TX0 < 2 ? 2 : TX0);   // pairs of lines per tile
  static constexpr int NTH = TX * TPC;
  static_assert(NTH <= 1024, "tile too large");
};

// twiddles e^{-2 pi i m/N}, m < N, each component broadcast to both lanes
template <int N, int NTH>
__device__ __forceinline__ void load_tw_pair(cpair* stw, const Tw& tw) {
  for (int q = threadIdx.x; q < N; q += NTH) {
    const float2 w = tw.f[N - 1 + q];
    stw[q] = cpair{make_float2(w.x, w.x), make_float2(w.y, w.y)};
  }
}

__device__ __forceinline__ cpair pair_of(float4 v) { return cpair{make_float2(v.x, v.z), make_float2(v.y, v.w)}; }
__device__ __forceinline__ float4 quad_of(cpair v) { return make_float4(v.x.x, v.y.x, v.x.y, v.y.y); }

template <int LOGN, int TX, int TPC, int SIGN, bool HALF = false>
__device__ __forceinline__ void col_body_pair(const AxisArgs& a, const Geo& g, const float2* in, float2* out,
                                              const Tw& tw, int item, unsigned char* smraw) {
  constexpr int N = 1 << LOGN;
  constexpr int NTH = TX * TPC;
  cpair* s = reinterpret_cast<cpair*>(smraw);
  cpair* stw = s + N * TX;
  const int r = item % a.nreal;
  const int tile = item / a.nreal;
  const int grp = tile / a.tpg;
  const int line = ((tile % a.tpg) * TX + (int)threadIdx.x % TX) * 2;
  const bool valid = line_valid(g, line, a.lines);
  const long long off = (long long)grp * a.gstride + line + (long long)r * a.rstride;
  const long long off0 = (long long)grp * a.gstride + (valid ? line : 0) + (long long)r * a.rstride;
  const float4* src = reinterpret_cast<const float4*>(in + off0);   // past the grid: line 0, nothing stored
  float4* dst = reinterpret_cast<float4*>(out + off);
  const int S2 = (int)(a.S / 2);   // stride in pairs: S is a multiple of the even row pitch
  const int nout = a.nout;
  constexpr int NR0 = N / Sched<LOGN>::radix(0);
  load_tw_pair<N, NTH>(stw, tw);
  __syncthreads();
  fft_tile<LOGN, TX, TPC, SIGN, TX, false, false, HALF>(
      s, stw,
      [&](int jb, int rr) { return pair_of(src[(jb + rr * NR0) * S2]); },
      [&](int pos, cpair v) {
        if (valid && pos < nout) dst[pos * S2] = quad_of(v);
      });
}

// synthesis + first inverse pass for two lines (indices i0 = even, i1 = i0 + 1
// of one row); the row state of a position serves both, the two amplitudes
// are one 8-byte load.  Decisions as in colgen_body.
template <int LOGN, int TX, int TPC, int GAUSS, bool HALF = false>
__device__ __forceinline__ void colgen_body_pair(const AxisArgs& a, const Geo& g, const float* __restrict__ amp,
                                                 const uint32_t* __restrict__ rowstates,
                                                 const uint32_t* __restrict__ apow, float2* out, const Tw& tw,
                                                 int item, unsigned char* smraw) {
  constexpr int N = 1 << LOGN;
  constexpr int NTH = TX * TPC;
  constexpr int R0 = Sched<LOGN>::radix(0);
  constexpr int NR0 = N / R0;
  cpair* s = reinterpret_cast<cpair*>(smraw);
  cpair* stw = s + N * TX;
  const int r = item % a.nreal;
  const int tile = item / a.nreal;
  const int grp = tile / a.tpg;
  const int line = ((tile % a.tpg) * TX + (int)threadIdx.x % TX) * 2;
  const bool valid = line_valid(g, line, a.lines);
  const int lsafe = valid ? line : 0;
  const bool zaxis = a.axis == 2;
  const int i0 = zaxis ? lsafe % g.HP : lsafe;
  const int i1 = i0 + 1;                     // may be the row padding (amplitude 0)
  const int j0 = zaxis ? lsafe / g.HP : 0;
  const int m = g.npx - 1;                   // npx is a power of two: indices wrap inside the table
  const uint32_t ai0 = __ldg(apow + (i0 & m)), aip0 = __ldg(apow + ((g.npx - i0) & m));
  const uint32_t ai1 = __ldg(apow + (i1 & m)), aip1 = __ldg(apow + ((g.npx - i1) & m));
  const bool iedge0 = (i0 == 0) || (2 * i0 == g.npx), iedge1 = 2 * i1 == g.npx;
  const int jp0 = (-j0) & (g.npy - 1);
  const bool cgt = zaxis && j0 > jp0;
  const bool selfrow = !zaxis || j0 == jp0;
  const bool self0 = selfrow && iedge0, self1 = selfrow && iedge1;
  const uint32_t* rs = rowstates + (size_t)r * g.npy * g.npz;
  const uint32_t* rs_own = rs + (zaxis ? (size_t)j0 * g.npz : 0);
  const uint32_t* rs_par = rs + (zaxis ? (size_t)jp0 * g.npz : 0);
  const long long cbase = (long long)grp * a.gstride + lsafe;
  const float2* ap = reinterpret_cast<const float2*>(amp + cbase);
  float4* dst = reinterpret_cast<float4*>(out + cbase + (long long)r * a.rstride);
  const int S2 = (int)(a.S / 2);
  const int nout = a.nout;
  load_tw_pair<N, NTH>(stw, tw);
  __syncthreads();
  fft_tile<LOGN, TX, TPC, +1, TX, false, false, HALF>(
      s, stw,
      [&](int jb, int rr) {
        const int p = jb + rr * NR0;
        const float2 am = __ldg(ap + p * S2);
        bool greater, mid;
        if (rr == 0) {
          mid = jb == 0;
          greater = mid && cgt;
        } else if (2 * rr == R0) {
          mid = jb == 0;
          greater = !mid || cgt;
        } else {
          mid = false;
          greater = 2 * rr > R0;
        }
        const uint32_t st = __ldg(partner_state(rs_own, rs_par, p, rr, greater, N));
        return coef_pair<GAUSS>(pm_mulmod(st, greater ? aip0 : ai0), pm_mulmod(st, greater ? aip1 : ai1), am,
                                mid && self0, mid && self1, greater);
      },
      [&](int pos, cpair v) {
        if (valid && pos < nout) dst[pos * S2] = quad_of(v);
      });
}

// ---------------------------------------------------------------- block reduction helpers
template <int NTH>
__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double red[2][NTH / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, off);
    b += __shfl_down_sync(0xffffffffu, b, off);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = a;
    red[1][threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s1 = 0, s2 = 0;
    for (int w = 0; w < NTH / 32; ++w) {
      s1 += red[0][w];
      s2 += red[1][w];
    }
    a = s1;
    b = s2;
  }
}

// ---------------------------------------------------------------- x pass: C2R + crop
// Row (j,k) of the half spectrum (N+1 values) -> npx = 2N reals, of which the
// first nx go to out[r][k][j][:].  Packing for a length-N inverse FFT:
//   Z[q] = (X[q] + conj X[N-q]) + i w^q (X[q] - conj X[N-q]),  w = e^{+2 pi i/(2N)}
// then x[2m] = Re z[m], x[2m+1] = Im z[m].  The imaginary parts of X[0] and
// X[N] are dropped: the reference keeps the real part of the full complex
// inverse (f90:1339), which does not see them.
template <typename R, int LOGN, int V = 0> struct RowCfg {
  using CF = ColCfg<R, LOGN, V>;
  static constexpr int N = CF::N, TPC = CF::TPC, ET = CF::ET;
  static constexpr int TX0 = CF::E / N;
  static constexpr int TX = TX0 > 64 ? 64 : (TX0 < 1 ? 1 : TX0);
  static constexpr int NTH0 = TX * TPC;
  static constexpr int NTH = NTH0 < 32 ? 32 : NTH0;
  static constexpr int PITCH = TX + 1;
};

// inverse length-N FFT of the TX rows staged in s (pitch TX+1), in place;
// twN holds e^{-2 pi i m/N}, m < N
template <typename R, int LOGN, int TX, int TPC>
__device__ __forceinline__ void fft_rows_inv(cpx_t<R>* s, const cpx_t<R>* twN) {
  using C = cpx_t<R>;
  constexpr int PITCH = TX + 1;
  static_assert(TX * TPC >= 32, "row tile needs at least one warp");
  if constexpr (LOGN > 0) {
    const int t = threadIdx.x % TX;
    constexpr int NR0 = (1 << LOGN) / Sched<LOGN>::radix(0);
    fft_tile<LOGN, TX, TPC, +1, PITCH, true, true>(
        s, twN, [&](int jb, int r) { return s[(jb + r * NR0) * PITCH + t]; },
        [&](int pos, C v) { s[pos * PITCH + t] = v; });
    __syncthreads();
  }
}

// part (may be NULL): per-block sums of x and x^2 for the mean/variance line
template <typename R, typename O, int LOGN, int TX, int TPC>
__device__ __forceinline__ void rows_body(const Geo& g, const cpx_t<R>* __restrict__ in, long long rstride,
                                          O* __restrict__ out, long long ostride, int nreal, int nblk_per_r,
                                          double* __restrict__ part, const Tw& tw, int item, unsigned char* smraw) {
  using C = cpx_t<R>;
  constexpr int N = 1 << LOGN, PITCH = TX + 1, NTH = TX * TPC;
  constexpr int NW = NTH / 32;
  C* s = reinterpret_cast<C*>(smraw);   // [N+1][PITCH]
  C* stw = s + (N + 1) * PITCH;         // 2N entries e^{-2 pi i m/(2N)}
  C* stwN = stw + 2 * N;                // N entries e^{-2 pi i m/N}
  const int r = item % nreal;
  const int blk = item / nreal;
  const int nrows = g.ny * g.nz;
  const int row0 = blk * TX;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = threadIdx.x; q < 2 * N; q += NTH) stw[q] = twtab<R>(tw)[2 * N - 1 + q];
  for (int q = threadIdx.x; q < N; q += NTH) stwN[q] = twtab<R>(tw)[N - 1 + q];
  const C* src = in + (long long)r * rstride;
  // stage rows: one warp per row, lanes along the row (coalesced)
  for (int t = warp; t < TX; t += NW) {
    const int row = row0 + t;
    const bool ok = row < nrows;
    const int j = ok ? row % g.ny : 0, k = ok ? row / g.ny : 0;
    const C* rp = src + ((long long)k * g.npy + j) * g.HP;
    constexpr int NIT = (N + 1 + 31) / 32;
    C tmp[NIT];
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int p = lane + 32 * it;
      tmp[it] = (ok && p <= N) ? rp[p] : cmk<C>(R(0), R(0));
    }
#pragma unroll
    for (int it = 0; it < NIT; ++it) {
      const int p = lane + 32 * it;
      if (p <= N) s[p * PITCH + t] = tmp[it];
    }
  }
  __syncthreads();
  // packing Z[q] from X[q], X[N-q], in place over the pairs (q, N-q)
  for (int q = threadIdx.x; q < (N / 2 + 1) * TX; q += NTH) {
    const int t = q % TX, k = q / TX;
    const int kc = N - k;
    C a = s[k * PITCH + t], b = s[kc * PITCH + t];
    if (k == 0) {
      a.y = R(0);
      b.y = R(0);
    }
    C w = stw[k];
    w.y = -w.y;
    const C bc = cmk<C>(b.x, -b.y);
    const C zk = cadd(cadd(a, bc), cmul_si<+1>(cmul(w, csub(a, bc))));
    if (k != 0 && kc != k) {
      C w2 = stw[kc];
      w2.y = -w2.y;
      const C ac = cmk<C>(a.x, -a.y);
      s[kc * PITCH + t] = cadd(cadd(b, ac), cmul_si<+1>(cmul(w2, csub(b, ac))));
    }
    s[k * PITCH + t] = zk;
  }
  __syncthreads();
  fft_rows_inv<R, LOGN, TX, TPC>(s, stwN);
  // write x[0..nx) of each row: one warp per row, lanes along m; FP64 sums for
  // the stats only when they are asked for (part != NULL, a uniform branch)
  double s1 = 0.0, s2 = 0.0;
  const bool stats = part != nullptr;
  O* dst = out + (long long)r * ostride;
  const int nxh = (g.nx + 1) / 2;
  const bool even = (g.nx & 1) == 0;
  for (int t = warp; t < TX; t += NW) {
    const int row = row0 + t;
    if (row >= nrows) break;
    O* rp = dst + (long long)row * g.nx;
    for (int m = lane; m < nxh; m += 32) {
      const C z = s[m * PITCH + t];
      const O a0 = (O)z.x, a1 = (O)z.y;
      const bool second = even || 2 * m + 1 < g.nx;
      if (even) {
        if constexpr (sizeof(O) == 4) {
          reinterpret_cast<float2*>(rp)[m] = make_float2((float)a0, (float)a1);
        } else {
          reinterpret_cast<double2*>(rp)[m] = make_double2((double)a0, (double)a1);
        }
      } else {
        rp[2 * m] = a0;
        if (second) rp[2 * m + 1] = a1;
      }
      if (stats) {
        s1 += (double)z.x;
        s2 += (double)z.x * (double)z.x;
        if (second) {
          s1 += (double)z.y;
          s2 += (double)z.y * (double)z.y;
        }
      }
    }
  }
  if (part) {
    block_sum2<NTH>(s1, s2);
    if (threadIdx.x == 0) {
      part[2 * ((long long)r * nblk_per_r + blk)] = s1;
      part[2 * ((long long)r * nblk_per_r + blk) + 1] = s2;
    }
  }
}

// ---------------------------------------------------------------- x pass, rows in warps
// The same C2R + crop with each row held by TPC lanes of one warp (RPW = 32 /
// TPC rows per warp): the N+1 inputs go from global memory straight into
// registers (lane rank c holds positions c + TPC i, coalesced), the packing
// takes X[N-q] from the mirrored lane by a shuffle, the transform runs on the
// warp's own shared-memory slice with warp barriers, and the last pass stores
// the cropped row.  Shared memory sees only the exchanges between radix passes
// (rows_body also stages the rows, packs in place and reads the result back).
// The packing and the butterflies are the operations of rows_body, so the
// values are the same bits.
template <typename R, int LOGN> struct RowWarpCfg {
  static constexpr int N = 1 << LOGN;
  static constexpr int ET = N > 256 ? 16 : 8;   // elements per lane
  static constexpr int TPC = N / ET;            // lanes per row
  static constexpr int RPW = TPC >= 32 ? 1 : 32 / TPC;
  static constexpr int NW = 8;                  // warps per block
  static constexpr int NTH = 32 * NW;
  static constexpr int ROWS = NW * RPW;         // rows per block
  static constexpr int SLICE = N * RPW;         // exchange elements per warp
  static constexpr bool ok = LOGN >= 3 && LOGN <= (sizeof(R) == 4 ? 9 : 8);
  static constexpr size_t smem = (size_t)(2 * N + NW * SLICE) * sizeof(cpx_t<R>);
};

template <typename R, typename O, int LOGN, bool HALF = false>
__device__ __forceinline__ void rows_warp_body(const Geo& g, const cpx_t<R>* __restrict__ in, long long rstride,
                                               O* __restrict__ out, long long ostride, int nreal, int nblk_per_r,
                                               double* __restrict__ part, const Tw& tw, int item,
                                               unsigned char* smraw) {
  using C = cpx_t<R>;
  using W = RowWarpCfg<R, LOGN>;
  constexpr int N = W::N, ET = W::ET, TPC = W::TPC, RPW = W::RPW;
  static_assert(W::ok && TPC * RPW == 32, "rows of whole warps");
  C* stw = reinterpret_cast<C*>(smraw);   // N entries e^{-2 pi i m/(2N)}
  C* stwN = stw + N;                      // N entries e^{-2 pi i m/N}
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  C* sx = stwN + N + warp * W::SLICE;
  const int r = item % nreal;
  const int blk = item / nreal;
  for (int q = threadIdx.x; q < N; q += W::NTH) {
    stw[q] = twtab<R>(tw)[2 * N - 1 + q];
    stwN[q] = twtab<R>(tw)[N - 1 + q];
  }
  const int t = lane % RPW, c = lane / RPW;
  const int nrows = g.ny * g.nz;
  const int row = (blk * W::NW + warp) * RPW + t;
  const bool ok = row < nrows;
  const int j = ok ? row % g.ny : 0, k = ok ? row / g.ny : 0;
  const C* rp = in + (long long)r * rstride + ((long long)k * g.npy + j) * g.HP;
  C x[ET];
#pragma unroll
  for (int i = 0; i < ET; ++i) x[i] = rp[c + TPC * i];
  const C xN = rp[N];
  __syncthreads();
  // Z[q] = (X[q] + conj X[N-q]) + i w^q (X[q] - conj X[N-q]), q = c + TPC i:
  // rank (TPC - c) of the row holds X[N-q] in register ET-1-i; rank 0 holds
  // X[N - TPC i] itself in register ET-i, and X[N]
  const int mirror = ((TPC - c) % TPC) * RPW + t;
  C z[ET];
#pragma unroll
  for (int i = 0; i < ET; ++i) {
    C b;
    b.x = __shfl_sync(0xffffffffu, x[ET - 1 - i].x, mirror);
    b.y = __shfl_sync(0xffffffffu, x[ET - 1 - i].y, mirror);
    if (c == 0) b = i == 0 ? xN : x[(ET - i) % ET];
    C a = x[i];
    const int q = c + TPC * i;
    if (q == 0) {
      a.y = R(0);
      b.y = R(0);
    }
    C w = stw[q];
    w.y = -w.y;
    const C bc = cmk<C>(b.x, -b.y);
    z[i] = cadd(cadd(a, bc), cmul_si<+1>(cmul(w, csub(a, bc))));
  }
  // pass-0 order of the engine: v[m R0 + r] = position c + TPC m + r N / R0
  constexpr int R0 = Sched<LOGN>::radix(0), NBT = ET / R0;
  C v[ET];
#pragma unroll
  for (int m = 0; m < NBT; ++m)
#pragma unroll
    for (int rr = 0; rr < R0; ++rr) v[m * R0 + rr] = z[m + rr * NBT];
  double s1 = 0.0, s2 = 0.0;
  const bool stats = part != nullptr;
  O* orow = out + (long long)r * ostride + (long long)(ok ? row : 0) * g.nx;
  const int nxh = (g.nx + 1) / 2;
  const bool even = (g.nx & 1) == 0;
  fft_tile_regs<LOGN, RPW, TPC, +1, RPW, false, false, -1, HALF>(sx, stwN, v, t, c, [&](int pos, C zz) {
    if (ok && pos < nxh) {
      const O a0 = (O)zz.x, a1 = (O)zz.y;
      const bool second = even || 2 * pos + 1 < g.nx;
      if (even) {
        if constexpr (sizeof(O) == 4) {
          reinterpret_cast<float2*>(orow)[pos] = make_float2((float)a0, (float)a1);
        } else {
          reinterpret_cast<double2*>(orow)[pos] = make_double2((double)a0, (double)a1);
        }
      } else {
        orow[2 * pos] = a0;
        if (second) orow[2 * pos + 1] = a1;
      }
      if (stats) {
        s1 += (double)zz.x;
        s2 += (double)zz.x * (double)zz.x;
        if (second) {
          s1 += (double)zz.y;
          s2 += (double)zz.y * (double)zz.y;
        }
      }
    }
  });
  if (part) {
    block_sum2<W::NTH>(s1, s2);
    if (threadIdx.x == 0) {
      part[2 * ((long long)r * nblk_per_r + blk)] = s1;
      part[2 * ((long long)r * nblk_per_r + blk) + 1] = s2;
    }
  }
}

// ---------------------------------------------------------------- x pass, two rows per lane on packed FP32
// Row variant 6 (FP32, lengths 8..256): rows_warp_body with the rows taken in
// pairs (A = 2 p, B = 2 p + 1), each lane holding one cpair per position (the
// real parts of A and B in one register pair, the imaginary parts in the
// other).  The packing and every butterfly and twiddle product is then one
// packed FP32 instruction for both rows, and the shuffles' lane arithmetic,
// the exchange addresses and the crop tests are shared by the two.  Lane by
// lane the operations are those of rows_warp_body (ksub on pairs is
// fma(b, -1, a), the exact IEEE difference), so the values are the same bits.
// The exchange layout of the row-warp tiles keeps its minimum number of
// shared-memory wavefronts with 16-byte elements.
template <int LOGN> struct RowPairCfg {
  static constexpr int N = 1 << LOGN;
  static constexpr int ET = 8;                  // pairs of elements per lane
  static constexpr int TPC = N / ET;            // lanes per row pair
  static constexpr int RPW = TPC >= 32 ? 1 : 32 / TPC;
  static constexpr int NW = 8;                  // warps per block
  static constexpr int NTH = 32 * NW;
  static constexpr int ROWS = 2 * NW * RPW;     // rows per block
  static constexpr int SLICE = N * RPW;         // exchange elements per warp
  static constexpr bool ok = LOGN >= 3 && LOGN <= 8;
  static constexpr size_t smem = (size_t)(2 * N + NW * SLICE) * sizeof(cpair);
};

__device__ __forceinline__ cpair pair_rows(float2 a, float2 b) {
  return cpair{make_float2(a.x, b.x), make_float2(a.y, b.y)};
}

template <typename O, int LOGN>
__device__ __forceinline__ void rows_pair_body(const Geo& g, const float2* __restrict__ in, long long rstride,
                                               O* __restrict__ out, long long ostride, int nreal, int nblk_per_r,
                                               double* __restrict__ part, const Tw& tw, int item,
                                               unsigned char* smraw) {
  using C = cpair;
  using W = RowPairCfg<LOGN>;
  constexpr int N = W::N, ET = W::ET, TPC = W::TPC, RPW = W::RPW;
  static_assert(W::ok && TPC * RPW == 32, "row pairs of whole warps");
  C* stw = reinterpret_cast<C*>(smraw);   // N entries e^{-2 pi i m/(2N)}, broadcast to both rows
  C* stwN = stw + N;                      // N entries e^{-2 pi i m/N}
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  C* sx = stwN + N + warp * W::SLICE;
  const int r = item % nreal;
  const int blk = item / nreal;
  for (int q = threadIdx.x; q < N; q += W::NTH) {
    const float2 a = tw.f[2 * N - 1 + q], b = tw.f[N - 1 + q];
    stw[q] = cpair{make_float2(a.x, a.x), make_float2(a.y, a.y)};
    stwN[q] = cpair{make_float2(b.x, b.x), make_float2(b.y, b.y)};
  }
  const int t = lane % RPW, c = lane / RPW;
  const int nrows = g.ny * g.nz;
  const int rowA = ((blk * W::NW + warp) * RPW + t) * 2, rowB = rowA + 1;
  const bool okA = rowA < nrows, okB = rowB < nrows;
  const int jA = okA ? rowA % g.ny : 0, kA = okA ? rowA / g.ny : 0;
  const int jB = okB ? rowB % g.ny : 0, kB = okB ? rowB / g.ny : 0;
  const float2* src = in + (long long)r * rstride;
  const float2* rpA = src + ((long long)kA * g.npy + jA) * g.HP;
  const float2* rpB = src + ((long long)kB * g.npy + jB) * g.HP;
  C x[ET];
#pragma unroll
  for (int i = 0; i < ET; ++i) x[i] = pair_rows(rpA[c + TPC * i], rpB[c + TPC * i]);
  const C xN = pair_rows(rpA[N], rpB[N]);
  __syncthreads();
  // the packing of rows_warp_body on both rows at once
  const int mirror = ((TPC - c) % TPC) * RPW + t;
  C z[ET];
#pragma unroll
  for (int i = 0; i < ET; ++i) {
    C b;
    b.x.x = __shfl_sync(0xffffffffu, x[ET - 1 - i].x.x, mirror);
    b.x.y = __shfl_sync(0xffffffffu, x[ET - 1 - i].x.y, mirror);
    b.y.x = __shfl_sync(0xffffffffu, x[ET - 1 - i].y.x, mirror);
    b.y.y = __shfl_sync(0xffffffffu, x[ET - 1 - i].y.y, mirror);
    if (c == 0) b = i == 0 ? xN : x[(ET - i) % ET];
    C a = x[i];
    const int q = c + TPC * i;
    if (q == 0) {
      a.y = make_float2(0.f, 0.f);
      b.y = make_float2(0.f, 0.f);
    }
    C w = stw[q];
    w.y = kneg(w.y);
    const C bc = cmk<C>(b.x, kneg(b.y));
    z[i] = cadd(cadd(a, bc), cmul_si<+1>(cmul(w, csub(a, bc))));
  }
  constexpr int R0 = Sched<LOGN>::radix(0), NBT = ET / R0;
  C v[ET];
#pragma unroll
  for (int m = 0; m < NBT; ++m)
#pragma unroll
    for (int rr = 0; rr < R0; ++rr) v[m * R0 + rr] = z[m + rr * NBT];
  double s1 = 0.0, s2 = 0.0;
  const bool stats = part != nullptr;
  O* orA = out + (long long)r * ostride + (long long)(okA ? rowA : 0) * g.nx;
  O* orB = out + (long long)r * ostride + (long long)(okB ? rowB : 0) * g.nx;
  const int nxh = (g.nx + 1) / 2;
  const bool even = (g.nx & 1) == 0;
  auto put = [&](O* orow, float re, float im, int pos) {
    const bool second = even || 2 * pos + 1 < g.nx;
    if (even) {
      if constexpr (sizeof(O) == 4) {
        reinterpret_cast<float2*>(orow)[pos] = make_float2(re, im);
      } else {
        reinterpret_cast<double2*>(orow)[pos] = make_double2((double)re, (double)im);
      }
    } else {
      orow[2 * pos] = (O)re;
      if (second) orow[2 * pos + 1] = (O)im;
    }
    if (stats) {
      s1 += (double)re;
      s2 += (double)re * (double)re;
      if (second) {
        s1 += (double)im;
        s2 += (double)im * (double)im;
      }
    }
  };
  fft_tile_regs<LOGN, RPW, TPC, +1, RPW, false, false, -1>(sx, stwN, v, t, c, [&](int pos, C zz) {
    if (pos < nxh) {
      if (okA) put(orA, zz.x.x, zz.y.x, pos);
      if (okB) put(orB, zz.x.y, zz.y.y, pos);
    }
  });
  if (part) {
    block_sum2<W::NTH>(s1, s2);
    if (threadIdx.x == 0) {
      part[2 * ((long long)r * nblk_per_r + blk)] = s1;
      part[2 * ((long long)r * nblk_per_r + blk) + 1] = s2;
    }
  }
}

}  // namespace ss3d
