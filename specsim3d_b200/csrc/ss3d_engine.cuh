// ss3d_engine.cuh -- register-resident Stockham FFT of a tile of TX columns.
//
// Thread layout: t = threadIdx.x % TX is the column, c = threadIdx.x / TX its
// rank among the TPC threads of that column.  Every thread owns ET = N / TPC
// elements in registers at all times.  The first radix pass reads its inputs
// straight from the loader (global memory or on-the-fly synthesis), the last
// pass hands its outputs straight to the storer; only the exchanges between
// passes go through shared memory (layout s[position * TX + t]).  For
// N = 512 = 8 * 8 * 8 this is two shared-memory round trips per element.
//
// Stockham indexing of pass p (radix R, Ns = product of earlier radices):
// butterfly jb reads positions jb + r*N/R, multiplies input r by
// w^(k*r), k = jb mod Ns, w = e^{SIGN 2 pi i/(Ns*R)}, applies the radix-R DFT
// and writes positions (jb/Ns)*Ns*R + k + r*Ns.  After the last pass the data
// are in natural order.
//
// Exchange layout: position p of column t sits at s[sw(p) * PITCH + t] with
// sw(p) = p ^ ((p >> 3) & SWM), a permutation inside each block of 8
// positions.  When a shared-memory row (PITCH elements) is narrower than the
// 128 bytes of the banks, the radix-8 stores of pass 0 (positions 8 jb + r,
// lanes differing in jb) would otherwise all fall into the same part of each
// bank row; the XOR spreads them over the whole row.  Reads, whose lanes take
// consecutive positions, keep touching the same addresses in another order.
#pragma once
#include "ss3d_device.cuh"

namespace ss3d {

template <int SWM> __device__ __forceinline__ int sw(int p) { return SWM ? p ^ ((p >> 3) & SWM) : p; }

// Exchange index of position p of column t.  SWM >= 0: sw(p) * PITCH + t.
// SWM < 0 (tiles of one warp, PITCH = TX rows of one warp): a = p * PITCH + t
// permuted as a ^ ((a >> 3) & 15), a bijection (bits 4-6 are kept, bits 0-3
// take bits 3-6 in); every exchange of the Stockham schedule then uses the
// minimum number of shared-memory wavefronts for transform lengths 32..512.
template <int PITCH, int SWM> __device__ __forceinline__ int xidx(int p, int t) {
  if constexpr (SWM < 0) {
    const int a = p * PITCH + t;
    return a ^ ((a >> 3) & 15);
  } else {
    return sw<SWM>(p) * PITCH + t;
  }
}

// barrier among the NTH threads of a tile: a warp barrier when the tile is
// one warp (the tiles of the warps of a block are then independent)
template <int NTH> __device__ __forceinline__ void tile_sync() {
  if constexpr (NTH <= 32)
    __syncwarp();
  else
    __syncthreads();
}

// SWM of a row of PITCH elements of EB bytes: 128 / row - 1 for a row of a
// power-of-two size below 128 bytes, else 0
template <int PITCH, int EB> struct Swizzle {
  static constexpr int row = PITCH * EB;
  static constexpr bool pow2 = (row & (row - 1)) == 0;
  static constexpr int M = (pow2 && row < 128) ? (128 / row > 8 ? 7 : 128 / row - 1) : 0;
};

template <int LOGN, int TX, int TPC, int SIGN, int P, int PITCH, bool STORE_SYNC, int SWM, bool HALF, typename C,
          class Store>
__device__ __forceinline__ void fft_tile_rest(C* __restrict__ s, const C* __restrict__ tw, C* v, int t, int c,
                                              Store&& store) {
  constexpr int N = 1 << LOGN;
  constexpr int NP = Sched<LOGN>::npass;
  if constexpr (P < NP) {
    constexpr int ET = N / TPC;
    constexpr int R = Sched<LOGN>::radix(P);
    constexpr int NS = Sched<LOGN>::ns_before(P);
    constexpr int NBT = ET / R;
#pragma unroll
    for (int m = 0; m < NBT; ++m) {
      const int jb = c + TPC * m;
#pragma unroll
      for (int r = 0; r < R; ++r) v[m * R + r] = s[xidx<PITCH, SWM>(jb + r * (N / R), t)];
    }
#pragma unroll
    for (int m = 0; m < NBT; ++m) {
      const int jb = c + TPC * m;
      const int k = jb % NS;
#pragma unroll
      for (int r = 1; r < R; ++r) v[m * R + r] = cmul_sgn(v[m * R + r], tw[(k * r) * (N / (NS * R))], SIGN > 0);
      dftR<R, SIGN>(&v[m * R]);
    }
    if constexpr (P == NP - 1) {
      if constexpr (STORE_SYNC) tile_sync<TX * TPC>();
#pragma unroll
      for (int m = 0; m < NBT; ++m) {
        const int jb = c + TPC * m;
        const int k = jb % NS;
        const int idxD = (jb / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r)
          if (!HALF || 2 * r < R) store(idxD + r * NS, v[m * R + r]);   // position < N/2 iff 2r < R
      }
    } else {
      tile_sync<TX * TPC>();
#pragma unroll
      for (int m = 0; m < NBT; ++m) {
        const int jb = c + TPC * m;
        const int k = jb % NS;
        const int idxD = (jb / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) s[xidx<PITCH, SWM>(idxD + r * NS, t)] = v[m * R + r];
      }
      tile_sync<TX * TPC>();
      fft_tile_rest<LOGN, TX, TPC, SIGN, P + 1, PITCH, STORE_SYNC, SWM, HALF>(s, tw, v, t, c, store);
    }
  }
}


// Passes of the tile from pass-0 inputs already in registers: v[m * R0 + r]
// holds position jb + r * N / R0, jb = c + TPC * m (R0 the radix of pass 0).
// t = column, c = rank of the thread in its column.  SWM: exchange layout
// (xidx).  LOAD_SYNC / STORE_SYNC as for fft_tile.
template <int LOGN, int TX, int TPC, int SIGN, int PITCH, bool LOAD_SYNC, bool STORE_SYNC, int SWM,
          bool HALF = false, typename C, class Store>
__device__ __forceinline__ void fft_tile_regs(C* __restrict__ s, const C* __restrict__ tw, C* v, int t, int c,
                                              Store&& store) {
  constexpr int N = 1 << LOGN;
  constexpr int ET = N / TPC;
  constexpr int NP = Sched<LOGN>::npass;
  static_assert(ET % 8 == 0 || N < 8, "each thread must own whole radix-8 butterflies");
  constexpr int R = Sched<LOGN>::radix(0);
  constexpr int NBT = ET / R;
#pragma unroll
  for (int m = 0; m < NBT; ++m) dftR<R, SIGN>(&v[m * R]);
  if constexpr (LOAD_SYNC) tile_sync<TX * TPC>();
  if constexpr (NP == 1) {
#pragma unroll
    for (int m = 0; m < NBT; ++m) {
      const int jb = c + TPC * m;
#pragma unroll
      for (int r = 0; r < R; ++r)
        if (!HALF || 2 * r < R) store(jb * R + r, v[m * R + r]);   // one pass: jb = 0, position r
    }
  } else {
#pragma unroll
    for (int m = 0; m < NBT; ++m) {
      const int jb = c + TPC * m;
#pragma unroll
      for (int r = 0; r < R; ++r) s[xidx<PITCH, SWM>(jb * R + r, t)] = v[m * R + r];
    }
    tile_sync<TX * TPC>();
    fft_tile_rest<LOGN, TX, TPC, SIGN, 1, PITCH, STORE_SYNC, SWM, HALF>(s, tw, v, t, c, store);
  }
}

// load(jb, r) returns the input at position jb + r * N / R0 (R0 the radix of
// pass 0); r is a constant after unrolling, so a loader can resolve anything
// that depends on which part of the transform the position lies in at compile
// time.  store(pos, v) receives the output at position pos.
// PITCH: shared-memory row pitch (>= TX).  LOAD_SYNC: barrier between the
// pass-0 loads and the pass-0 shared-memory writes (loader reads s).
// STORE_SYNC: barrier before the final stores (storer writes s).
// HALF: the storer keeps only positions below N/2 (a pruned transform whose
// kept outputs all lie there); store is not called for the others, so the
// arithmetic that only feeds them is dropped at compile time, and the kept
// outputs are computed by the same operations as without HALF.
template <int LOGN, int TX, int TPC, int SIGN, int PITCH = TX, bool LOAD_SYNC = false, bool STORE_SYNC = false,
          bool HALF = false, typename C, class Load, class Store>
__device__ __forceinline__ void fft_tile(C* __restrict__ s, const C* __restrict__ tw, Load&& load, Store&& store) {
  constexpr int N = 1 << LOGN;
  constexpr int ET = N / TPC;
  constexpr int SWM = Swizzle<PITCH, (int)sizeof(C)>::M;
  const int t = threadIdx.x % TX;
  const int c = threadIdx.x / TX;
  C v[ET > 0 ? ET : 1];
  constexpr int R = Sched<LOGN>::radix(0);
  constexpr int NBT = ET / R;
#pragma unroll
  for (int m = 0; m < NBT; ++m) {
    const int jb = c + TPC * m;
#pragma unroll
    for (int r = 0; r < R; ++r) v[m * R + r] = load(jb, r);   // position jb + r * N / R
  }
  fft_tile_regs<LOGN, TX, TPC, SIGN, PITCH, LOAD_SYNC, STORE_SYNC, SWM, HALF>(s, tw, v, t, c, store);
}

}  // namespace ss3d
