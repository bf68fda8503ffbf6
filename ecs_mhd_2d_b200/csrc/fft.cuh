// Warp-level radix-2 FFTs of length N in {64, 128, 256} (one transform per warp).
//
// Data distribution: lane l holds E = N/32 complex values v[j] at "positions"
// e = l + 32*j.  Stages whose butterfly span is >= 32 are register-local; the
// five stages with span < 32 exchange values with __shfl_xor_sync.
//
//  * fft_dif : natural-order input  -> bit-reversed output (position e holds X[bitrev(e)])
//  * fft_dit : bit-reversed input   -> natural-order output
//
// Both are unnormalised.  FWD uses exp(-2 pi i k/N), INV uses exp(+2 pi i k/N).
// Twiddles come from a table tw[k] = exp(-2 pi i k / N), k in [0, N/2),
// computed on the host in long double and staged in shared memory.
#pragma once

#include "common.cuh"

namespace ecs {

template <int N> struct Log2E;
template <> struct Log2E<64>  { static constexpr int v = 1; };
template <> struct Log2E<128> { static constexpr int v = 2; };
template <> struct Log2E<256> { static constexpr int v = 3; };

template <typename R, bool INV>
__device__ __forceinline__ cplx<R> twid(const cplx<R>* __restrict__ tw, int idx) {
  cplx<R> w = tw[idx];
  if (INV) w.y = -w.y;
  return w;
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dif(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  constexpr int E = N / 32;
  constexpr int LE = Log2E<N>::v;
  // register stages: span s = 32*half, half = E/2 ... 1
#pragma unroll
  for (int m = LE - 1; m >= 0; --m) {
    const int half = 1 << m;
    const int s = 32 * half;
    const int stride = N / (2 * s);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if ((j & half) == 0) {
        cplx<R> a = v[j], b = v[j + half];
        v[j] = cadd(a, b);
        const int idx = (lane + 32 * (j & (half - 1))) * stride;
        v[j + half] = cmul(csub(a, b), twid<R, INV>(tw, idx));
      }
    }
  }
  // shuffle stages: span 16 ... 1
#pragma unroll
  for (int s = 16; s >= 1; s >>= 1) {
    const cplx<R> w = twid<R, INV>(tw, (lane & (s - 1)) * (N / (2 * s)));
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      cplx<R> p = shfl_xor_c<R>(v[j], s);
      v[j] = upper ? cmul(csub(p, v[j]), w) : cadd(v[j], p);
    }
  }
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dit(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  constexpr int E = N / 32;
  constexpr int LE = Log2E<N>::v;
#pragma unroll
  for (int s = 1; s <= 16; s <<= 1) {
    const cplx<R> w = twid<R, INV>(tw, (lane & (s - 1)) * (N / (2 * s)));
    const bool upper = (lane & s) != 0;
#pragma unroll
    for (int j = 0; j < E; ++j) {
      cplx<R> p = shfl_xor_c<R>(v[j], s);
      v[j] = upper ? csub(p, cmul(v[j], w)) : cadd(v[j], cmul(p, w));
    }
  }
#pragma unroll
  for (int m = 0; m < LE; ++m) {
    const int half = 1 << m;
    const int s = 32 * half;
    const int stride = N / (2 * s);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if ((j & half) == 0) {
        const int idx = (lane + 32 * (j & (half - 1))) * stride;
        cplx<R> b = cmul(v[j + half], twid<R, INV>(tw, idx));
        cplx<R> a = v[j];
        v[j] = cadd(a, b);
        v[j + half] = csub(a, b);
      }
    }
  }
}

// Cooperative copy of the N/2-entry twiddle table into shared memory.
template <typename R, int N>
__device__ __forceinline__ void load_twiddles(cplx<R>* s_tw, const cplx<R>* __restrict__ g_tw) {
  for (int i = threadIdx.x; i < N / 2; i += blockDim.x) s_tw[i] = g_tw[i];
}

}  // namespace ecs
