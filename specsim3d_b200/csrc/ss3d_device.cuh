// ss3d_device.cuh -- device-side building blocks shared by the SPECSIM3D
// kernels: complex helpers, the Park-Miller jump-ahead stream, the Hermitian
// draw-offset arithmetic and the shared-memory Stockham FFT engine.
//
// Reference behaviour reproduced here (src/specsim3d.f90):
//   * urand / gauss_pair  f90:191-205  (Lehmer 16807 mod 2^31-1, Box-Muller)
//   * seeding             f90:1302-1303 (s0 = mod(|iseed|, 2^31-2) + 1, 10 draws)
//   * Hermitian fill      f90:1305-1334 (draw order k, j, i over lin <= linp)
//   * fft1d / fft3d       f90:208-304   (unscaled; isign -1 forward, +1 inverse)
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ss3d {

constexpr uint32_t PM_M = 2147483647u;  // 2^31 - 1
constexpr uint32_t PM_A = 16807u;

// ---------------------------------------------------------------- complex
// Three complex types share one set of operations, written once over the
// component type K of C::x and C::y:
//   double2  K = double  (FP64 path)
//   float2   K = float   (FP32, one column per thread)
//   cpair    K = float2  (FP32, two adjacent columns per thread: x holds the
//                          real parts of both, y the imaginary parts)
// For float and float2 every component operation is one explicitly rounded
// IEEE operation (no contraction left to the compiler), and cpair runs the
// packed sm_100 forms of the same operations lane by lane, so a transform
// gives the same bits in either FP32 layout.
struct __align__(16) cpair {
  float2 x, y;
};

template <typename R> struct cpx;
template <> struct cpx<float> { using T = float2; };
template <> struct cpx<double> { using T = double2; };
template <typename R> using cpx_t = typename cpx<R>::T;

__device__ __forceinline__ double kadd(double a, double b) { return a + b; }
__device__ __forceinline__ double ksub(double a, double b) { return a - b; }
__device__ __forceinline__ double kmul(double a, double b) { return a * b; }
__device__ __forceinline__ double kfma(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ double kneg(double a) { return -a; }
__device__ __forceinline__ float kadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float ksub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float kmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float kfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ float kneg(float a) { return -a; }
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
__device__ __forceinline__ float2 kadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 kmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 kfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
#else
__device__ __forceinline__ float2 kadd(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 kmul(float2 a, float2 b) { return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)); }
__device__ __forceinline__ float2 kfma(float2 a, float2 b, float2 c) {
  return make_float2(__fmaf_rn(a.x, b.x, c.x), __fmaf_rn(a.y, b.y, c.y));
}
#endif
__device__ __forceinline__ float2 kneg(float2 a) { return make_float2(-a.x, -a.y); }
// a - b = fma(b, -1, a): the product is exact, so this is the IEEE difference
__device__ __forceinline__ float2 ksub(float2 a, float2 b) { return kfma(b, make_float2(-1.f, -1.f), a); }

template <typename K> __device__ __forceinline__ K kconst(double v);
template <> __device__ __forceinline__ double kconst<double>(double v) { return v; }
template <> __device__ __forceinline__ float kconst<float>(double v) { return (float)v; }
template <> __device__ __forceinline__ float2 kconst<float2>(double v) { return make_float2((float)v, (float)v); }

template <typename C> using comp_t = decltype(C::x);
template <typename C> __device__ __forceinline__ C cmk(comp_t<C> a, comp_t<C> b) { C c; c.x = a; c.y = b; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(kadd(a.x, b.x), kadd(a.y, b.y)); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(ksub(a.x, b.x), ksub(a.y, b.y)); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return cmk<C>(kfma(kneg(a.y), b.y, kmul(a.x, b.x)), kfma(a.y, b.x, kmul(a.x, b.y)));
}
// a * b, or a * conj(b) when conjb is true
template <typename C> __device__ __forceinline__ C cmul_sgn(C a, C b, bool conjb) {
  if (conjb) return cmk<C>(kfma(a.y, b.y, kmul(a.x, b.x)), kfma(kneg(a.x), b.y, kmul(a.y, b.x)));
  return cmul(a, b);
}
// a + s i b and a - s i b, s = SIGN (multiplication by +-i is exact)
template <int SIGN, typename C> __device__ __forceinline__ C caddi(C a, C b) {
  return SIGN > 0 ? cmk<C>(ksub(a.x, b.y), kadd(a.y, b.x)) : cmk<C>(kadd(a.x, b.y), ksub(a.y, b.x));
}
template <int SIGN, typename C> __device__ __forceinline__ C csubi(C a, C b) {
  return SIGN > 0 ? cmk<C>(kadd(a.x, b.y), ksub(a.y, b.x)) : cmk<C>(ksub(a.x, b.y), kadd(a.y, b.x));
}
// multiply by (sign * i): forward (sign -1) gives -i, inverse gives +i
template <int SIGN, typename C> __device__ __forceinline__ C cmul_si(C a) {
  return SIGN > 0 ? cmk<C>(kneg(a.y), a.x) : cmk<C>(a.y, kneg(a.x));
}

// ---------------------------------------------------------------- Park-Miller
__host__ __device__ __forceinline__ uint32_t pm_mulmod(uint32_t a, uint32_t b) {
  // a, b < 2^31: p = a b < 2^62 = hi 2^32 + lo;  p mod (2^31 - 1) = (p & m) + (p >> 31) folded once
#ifdef __CUDA_ARCH__
  const uint32_t lo = a * b, hi = __umulhi(a, b);
#else
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  const uint32_t lo = (uint32_t)p, hi = (uint32_t)(p >> 32);
#endif
  uint32_t r = (lo & PM_M) + ((hi << 1) | (lo >> 31));   // <= 2m - 2 for a, b < m
  // r - m wraps above r when r < m: the unsigned minimum is the reduced value
#ifdef __CUDA_ARCH__
  return min(r, r - PM_M);
#else
  return r >= PM_M ? r - PM_M : r;
#endif
}

// the same product without the final conditional subtraction: a value in
// [0, 2m) congruent to a b (mod m), for consumers that accept either
// representative (the FP32 phase reduction below)
__host__ __device__ __forceinline__ uint32_t pm_mulmod_lazy(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
  const uint32_t lo = a * b, hi = __umulhi(a, b);
#else
  const uint64_t p = (uint64_t)a * (uint64_t)b;
  const uint32_t lo = (uint32_t)p, hi = (uint32_t)(p >> 32);
#endif
  return (lo & PM_M) + ((hi << 1) | (lo >> 31));
}

// 16807^e mod (2^31-1) from the three 11-bit power tables
// tab[l*2048 + v] = 16807^(v * 2048^l) mod m, e < 2^31 (reduced mod m-1).
__device__ __forceinline__ uint32_t pm_pow(const uint32_t* __restrict__ tab, uint64_t e) {
  e %= (uint64_t)(PM_M - 1);
  uint32_t r = tab[e & 2047u];
  r = pm_mulmod(r, tab[2048 + ((e >> 11) & 2047u)]);
  r = pm_mulmod(r, tab[4096 + ((e >> 22) & 2047u)]);
  return r;
}

// ---------------------------------------------------------------- grid geometry
// Padded periodic grid (npx, npy, npz) and the Hermitian half spectrum
// i in [0, H), H = npx/2 + 1 (1 when npx = 1), stored with row pitch HP.
struct Geo {
  int npx, npy, npz;   // periodic grid
  int nx, ny, nz;      // output grid
  int H, HP;           // half-spectrum width and row pitch (elements)
  int d;               // draws per representative index (1 phases, 2 Gaussian)
  uint64_t D;          // draws per realization
};

// number of representative indices (lin <= linp) in the rows of plane k that
// precede row j, plus all planes before k  (row order k, j as in f90:1306-1308)
__host__ __device__ __forceinline__ uint64_t row_prefix(const Geo& g, int j, int k) {
  const uint64_t npx = g.npx, npy = g.npy;
  const uint64_t Hr = g.npx >= 2 ? (uint64_t)(g.npx / 2 + 1) : 1u;
  const uint64_t nless_rows = g.npy >= 2 ? (uint64_t)(g.npy / 2 - 1) : 0u;
  const uint64_t neq_rows = g.npy >= 2 ? 2u : 1u;
  const uint64_t qeq = nless_rows * npx + neq_rows * Hr;   // count of a self-conjugate plane
  uint64_t P = 0;
  if (k > 0) {
    P = qeq;
    if (g.npz >= 2) {
      int half = g.npz / 2;
      int full = (k < half ? k : half) - 1;
      if (full > 0) P += (uint64_t)full * npy * npx;
      if (k > half) P += qeq;
    }
  }
  const int kp = (g.npz - k) % g.npz;
  if (k < kp) return P + (uint64_t)j * npx;
  if (k > kp) return P;
  if (j == 0) return P;
  uint64_t s = Hr;
  if (g.npy >= 2) {
    int half = g.npy / 2;
    s += (uint64_t)((j < half ? j : half) - 1) * npx;
    if (j > half) s += Hr;
  }
  return P + s;
}

// class of row (j,k): 0 all indices are representatives, 1 self-conjugate row
// (i <= npx/2 are representatives), 2 none (conjugates of row (jp,kp))
__host__ __device__ __forceinline__ int row_class(const Geo& g, int j, int k) {
  const int jp = (g.npy - j) % g.npy, kp = (g.npz - k) % g.npz;
  if (k < kp || (k == kp && j < jp)) return 0;
  if (k > kp || (k == kp && j > jp)) return 2;
  return 1;
}

// ---------------------------------------------------------------- coefficient synthesis
// Hardware approximations of the PTX ISA (sin.approx, cos.approx, lg2.approx,
// rsqrt.approx, rcp.approx; .ftz: every argument below is a normal number),
// issued directly so that no range or subnormal handling is added around them.
__device__ __forceinline__ float sin_hw(float x) { float r; asm("sin.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
__device__ __forceinline__ float cos_hw(float x) { float r; asm("cos.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
__device__ __forceinline__ float lg2_hw(float x) { float r; asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
__device__ __forceinline__ float rsqrt_hw(float x) { float r; asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }
__device__ __forceinline__ float rcp_hw(float x) { float r; asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x)); return r; }

// Unit phasor e^{2 pi i s/m} in float, for any s < 2m congruent to the state
// (mod m).  The nearest half turn n of 2s/m is taken in integers from
// s / 2^30 (which differs from 2s/m by less than 2^-29 relative, so n is the
// nearest half turn or, at a boundary, its neighbour), and the remainder
// 2s - n m is exact in 32-bit modular arithmetic; |x| <= pi/2 + 1e-8 (argument
// error about 1e-7: one float rounding of the exact integer remainder) goes
// through the hardware sine and cosine (absolute error about 2^-21), and odd
// half turns negate both (s and s - m give half turns of the same parity).
// Half of the phases use the hardware values with each sign, so their small
// systematic error averages out over a spectrum instead of adding up
// coherently: a reduction to [-pi, pi] without the alternating sign left a
// bias that summed to 4e-5 sqrt(C0) at the cell where every phase is 1 (the
// origin) on a 512^3 spectrum.
__device__ __forceinline__ int half_turns(uint32_t s) { return (int)((s >> 30) + ((s >> 29) & 1u)); }
__device__ __forceinline__ int half_turn_rem(uint32_t s, int n) {
  return (int)(2u * s - ((uint32_t)n << 31) + (uint32_t)n);   // 2s - n (2^31 - 1)  (mod 2^32)
}
// cos and sin of the remainder; returns true for an odd half-turn count, when
// the phasor is (-c, -sn): callers fold that sign into their scale factor
__device__ __forceinline__ bool phasor_half_f(uint32_t s, float& c, float& sn) {
  const int n = half_turns(s);
  const float x = (float)half_turn_rem(s, n) * 1.4629181e-9f;   // pi / (2^31-1)
  sn = sin_hw(x);
  c = cos_hw(x);
  return n & 1;
}
__device__ __forceinline__ void phasor_d(uint32_t s, double& c, double& sn) {
  double u = (double)s / 2147483647.0;
  sincospi(2.0 * u, &sn, &c);
}
// -2 ln(s/m) in float for s in [1, m-1].  For u = s/m >= 3/4 the logarithm is
// 2 atanh(z), z = (u-1)/(u+1) = -(m-s)/(m+s) with |z| <= 1/7, from the exact
// integer difference m-s (odd series to z^7, truncation below 2e-8 relative;
// the quotient by the hardware reciprocal, relative error about 2^-23);
// below 3/4 |ln u| >= 0.28 and the hardware log2 (absolute error ~2^-22) is
// accurate to a few 1e-7 relative.
// The series is evaluated as q (4 + 4/3 q^2 + 4/5 q^4 + 4/7 q^6), q = -z; the far
// branch as -2 ln 2 (log2 s - 31), u = s 2^-31 (the float of 1/(2^31 - 1)).
constexpr float M2LOG_C31 = 42.975124f;   // 2 ln 2 * 31
__device__ __forceinline__ float m2log_f(uint32_t s) {
  const float a = (float)(PM_M - s);
  const float q = a * rcp_hw(4294967294.0f - a);           // -z = (1-u)/(1+u), m + s = 2m - (m - s)
  const float z2 = q * q;
  float p = fmaf(z2, 4.0f / 7.0f, 4.0f / 5.0f);
  p = fmaf(z2, p, 4.0f / 3.0f);
  p = fmaf(z2, p, 4.0f);
  const float near1 = p * q;
  const float far = fmaf(-1.3862944f, lg2_hw((float)s), M2LOG_C31);
  return s >= 1610612736u ? near1 : far;                    // u >= 3/4
}
__device__ __forceinline__ double m2log_d(uint32_t s) {
  double u = (double)s / 2147483647.0;
  return -2.0 * log(u);
}

// Park-Miller state right after the first draw that produced coefficient
// (i, j, k): the index itself for representative rows, its conjugate partner
// (ip, jp, kp) for rows of class 2 (conj = true).  self marks the
// self-conjugate indices (lin == linp).
__device__ __forceinline__ uint32_t first_state(const Geo& g, int i, int j, int k, const uint32_t* __restrict__ rs,
                                                const uint32_t* __restrict__ apow, bool& conj, bool& self) {
  int cls = row_class(g, j, k);
  int si = i, sj = j, sk = k;
  conj = false;
  if (cls == 2) {
    si = (g.npx - i) % g.npx;
    sj = (g.npy - j) % g.npy;
    sk = (g.npz - k) % g.npz;
    conj = true;
  }
  self = (cls == 1) && (i == 0 || 2 * i == g.npx);
  return pm_mulmod(rs[(size_t)sj * g.npz + sk], apow[si]);   // row states [j][k]
}

// Coefficient of half-spectrum index (i, j, k) for the realization whose row
// states are rs (state of the first draw of each row of the realization).
// Reproduces f90:1312-1331 for the half spectrum:
//   row class 0 (or self-conjugate row, non-self index): amp * (g1 + i g2) sqrt(1/2)
//     or amp * e^{i phi}
//   row class 2: conjugate of the partner draw at (ip, jp, kp)
//   self-conjugate index: amp * g1 (Gaussian) or +/-amp (phases, u < 0.5 -> +)
template <typename R>
__device__ __forceinline__ cpx_t<R> coefficient(const Geo& g, int i, int j, int k, R amp,
                                                 const uint32_t* __restrict__ rs,
                                                 const uint32_t* __restrict__ apow) {
  using C = cpx_t<R>;
  bool conj, self;
  uint32_t s1 = first_state(g, i, j, k, rs, apow, conj, self);
  if (g.d == 2) {
    const uint32_t s2 = sizeof(R) == 4 ? pm_mulmod_lazy(s1, PM_A) : pm_mulmod(s1, PM_A);
    if constexpr (sizeof(R) == 4) {
      const float L = m2log_f(s1);
      float rr = L * rsqrt_hw(L);
      float cs, sn;
      const bool odd = phasor_half_f(s2, cs, sn);
      const float t0 = (self ? amp : amp * 0.70710678118654752f) * rr;
      const float t = odd ? -t0 : t0;
      if (self) return cmk<C>(t * cs, 0.f);
      return cmk<C>(t * cs, (conj ? -t : t) * sn);
    } else {
      double rr = sqrt(m2log_d(s1));
      double cs, sn;
      phasor_d(s2, cs, sn);
      double g1 = rr * cs, g2 = rr * sn;
      if (self) return cmk<C>(amp * g1, 0.0);
      const double h = 0.70710678118654757;   // sqrt(0.5d0)
      return cmk<C>(amp * g1 * h, amp * (conj ? -g2 : g2) * h);
    }
  } else {
    if (self) {
      // urand() < 0.5  <=>  s/m < 0.5 with s integer  <=>  2 s < m
      bool pos = (2ull * s1) < (uint64_t)PM_M;
      return cmk<C>(pos ? amp : -amp, R(0));
    }
    R cs, sn, a = amp;
    if constexpr (sizeof(R) == 4) {
      if (phasor_half_f(s1, cs, sn)) a = -a;
    } else {
      phasor_d(s1, cs, sn);
    }
    return cmk<C>(a * cs, conj ? -(a * sn) : a * sn);
  }
}

// Coefficient of index (i, j, k) with the index-i dependent parts precomputed
// by the caller: ai = 16807^(d i), aip = 16807^(d ((npx - i) mod npx)),
// iedge = (i == 0 or 2 i == npx).  Same values as coefficient().
template <typename R>
__device__ __forceinline__ cpx_t<R> coef_col(const Geo& g, int j, int k, R amp, const uint32_t* __restrict__ rs,
                                             uint32_t ai, uint32_t aip, bool iedge) {
  using C = cpx_t<R>;
  const int jp = (-j) & (g.npy - 1), kp = (-k) & (g.npz - 1);
  const bool less = k < kp || (k == kp && j < jp);
  const bool greater = k > kp || (k == kp && j > jp);
  const int row = greater ? jp * g.npz + kp : j * g.npz + k;   // row states [j][k]
  const uint32_t s1 = pm_mulmod(__ldg(rs + row), greater ? aip : ai);
  const bool self = !less && !greater && iedge;
  if (g.d == 2) {
    const uint32_t s2 = sizeof(R) == 4 ? pm_mulmod_lazy(s1, PM_A) : pm_mulmod(s1, PM_A);
    if constexpr (sizeof(R) == 4) {
      const float L = m2log_f(s1);
      const float rr = L * rsqrt_hw(L);
      float cs, sn;
      const bool odd = phasor_half_f(s2, cs, sn);
      const float t0 = (self ? amp : amp * 0.70710678118654752f) * rr;
      const float t = odd ? -t0 : t0;
      if (self) return cmk<C>(t * cs, 0.f);
      return cmk<C>(t * cs, (greater ? -t : t) * sn);
    } else {
      const double rr = sqrt(m2log_d(s1));
      double cs, sn;
      phasor_d(s2, cs, sn);
      const double g1 = rr * cs, g2 = rr * sn;
      if (self) return cmk<C>(amp * g1, 0.0);
      const double h = 0.70710678118654757;
      return cmk<C>(amp * g1 * h, amp * (greater ? -g2 : g2) * h);
    }
  } else {
    if (self) return cmk<C>((2ull * s1) < (uint64_t)PM_M ? amp : -amp, R(0));
    R cs, sn, a = amp;
    if constexpr (sizeof(R) == 4) {
      if (phasor_half_f(s1, cs, sn)) a = -a;
    } else {
      phasor_d(s1, cs, sn);
    }
    return cmk<C>(a * cs, greater ? -(a * sn) : a * sn);
  }
}

// ---------------------------------------------------------------- small DFTs
template <int SIGN, typename C> __device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a; a = cadd(t, b); b = csub(t, b);
}
template <int SIGN, typename C> __device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
  C t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), d = csub(v1, v3);
  v0 = cadd(t0, t2); v2 = csub(t0, t2); v1 = caddi<SIGN>(t1, d); v3 = csubi<SIGN>(t1, d);
}
// radix 8 as two radix 4 and the w8 combination.  With w8 = (1 + s i)/sqrt(2),
// q = (x + y)/sqrt(2) and u = (x - y)/sqrt(2) of o = (x, y):
//   s = +1:  o w8 = (u, q),   o w8^3 = (-q, u)
//   s = -1:  o w8 = (q, -u),  o w8^3 = (-u, -q)
template <int SIGN, typename C> __device__ __forceinline__ void dft8(C* v) {
  using K = comp_t<C>;
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<SIGN>(e0, e1, e2, e3);
  dft4<SIGN>(o0, o1, o2, o3);
  const K r2 = kconst<K>(0.70710678118654752440);
  const K q1 = kmul(kadd(o1.x, o1.y), r2), u1 = kmul(ksub(o1.x, o1.y), r2);
  const K q3 = kmul(kadd(o3.x, o3.y), r2), u3 = kmul(ksub(o3.x, o3.y), r2);
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[2] = caddi<SIGN>(e2, o2); v[6] = csubi<SIGN>(e2, o2);
  if constexpr (SIGN > 0) {
    v[1] = cmk<C>(kadd(e1.x, u1), kadd(e1.y, q1)); v[5] = cmk<C>(ksub(e1.x, u1), ksub(e1.y, q1));
    v[3] = cmk<C>(ksub(e3.x, q3), kadd(e3.y, u3)); v[7] = cmk<C>(kadd(e3.x, q3), ksub(e3.y, u3));
  } else {
    v[1] = cmk<C>(kadd(e1.x, q1), ksub(e1.y, u1)); v[5] = cmk<C>(ksub(e1.x, q1), kadd(e1.y, u1));
    v[3] = cmk<C>(ksub(e3.x, u3), ksub(e3.y, q3)); v[7] = cmk<C>(kadd(e3.x, u3), kadd(e3.y, q3));
  }
}
template <int R, int SIGN, typename C> __device__ __forceinline__ void dftR(C* v) {
  if constexpr (R == 8) dft8<SIGN>(v);
  else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
}

// radix of pass number p for a length 2^LOGN transform: radix-8 passes first,
// then one radix-4 or radix-2 pass for the remaining bits
template <int LOGN> struct Sched {
  static constexpr int n8 = LOGN / 3;
  static constexpr int rem = LOGN % 3;
  static constexpr int npass = n8 + (rem ? 1 : 0);
  static constexpr int radix(int p) { return p < n8 ? 8 : (rem == 2 ? 4 : 2); }
  static constexpr int ns_before(int p) { return p == 0 ? 1 : ns_before(p - 1) * radix(p - 1); }
};

// One Stockham pass (Ns = sub-transform size already done, R = radix) over a
// tile stored in shared memory as s[p * PITCH + t], t in [0,TX) columns,
// p in [0,N) positions.  In place: every item is loaded before the barrier and
// stored after it.  tw: shared twiddles, tw[m] = e^{-2 pi i m / N}.
template <int N, int TX, int PITCH, int NT, int R, int NS, int SIGN, int TWS, typename C>
__device__ __forceinline__ void stockham_pass(C* s, const C* tw) {
  constexpr int NB = N / R;                 // butterflies per column
  constexpr int TOTAL = NB * TX;
  constexpr int ITEMS = (TOTAL + NT - 1) / NT;
  C v[ITEMS][R];
#pragma unroll
  for (int it = 0; it < ITEMS; ++it) {
    int q = it * NT + (int)threadIdx.x;
    if (TOTAL % NT == 0 || q < TOTAL) {
      int t = q % TX, jb = q / TX;
      int k = jb % NS;
#pragma unroll
      for (int r = 0; r < R; ++r) v[it][r] = s[(jb + r * NB) * PITCH + t];
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = tw[(k * r) * (N / (NS * R)) * TWS];
          v[it][r] = cmul_sgn(v[it][r], w, SIGN > 0);
        }
      }
      dftR<R, SIGN>(v[it]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int it = 0; it < ITEMS; ++it) {
    int q = it * NT + (int)threadIdx.x;
    if (TOTAL % NT == 0 || q < TOTAL) {
      int t = q % TX, jb = q / TX;
      int k = jb % NS;
      int idxD = (jb / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[(idxD + r * NS) * PITCH + t] = v[it][r];
    }
  }
  __syncthreads();
}

template <int N, int TX, int PITCH, int NT, int SIGN, int TWS, int LOGN, int P, typename C>
__device__ __forceinline__ void stockham_from(C* s, const C* tw) {
  if constexpr (P < Sched<LOGN>::npass) {
    stockham_pass<N, TX, PITCH, NT, Sched<LOGN>::radix(P), Sched<LOGN>::ns_before(P), SIGN, TWS>(s, tw);
    stockham_from<N, TX, PITCH, NT, SIGN, TWS, LOGN, P + 1>(s, tw);
  }
}

// Full length-2^LOGN transform of TX columns in shared memory (unscaled).
// tw[m * TWS] = e^{-2 pi i m / 2^LOGN}.  Caller must __syncthreads() after
// filling s and tw; the transform ends with a barrier.
template <int LOGN, int TX, int PITCH, int NT, int SIGN, int TWS = 1, typename C>
__device__ __forceinline__ void smem_fft(C* s, const C* tw) {
  stockham_from<(1 << LOGN), TX, PITCH, NT, SIGN, TWS, LOGN, 0>(s, tw);
}

}  // namespace ss3d
