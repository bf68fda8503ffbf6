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
// computed on the host in long double.  In shared memory it is expanded to one
// contiguous sub-table per index stride r = 1, 2, 4, ...:
//   s_tw[tw_off(N, r) + i] = tw[i r],  i < N / (2 r),  tw_off(N, r) = N - N / r,
// so that every stage reads consecutive entries across lanes (a strided read
// of the plain table hits the same shared-memory banks from several lanes).
#pragma once

#include "common.cuh"

namespace ecs {

// Shared-memory twiddle entries and the offset of the stride-r sub-table.
__host__ __device__ constexpr int tw_smem(int N) { return N; }
__host__ __device__ constexpr int tw_off(int N, int r) { return N - N / r; }

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

// Multiply by -i (forward) or +i (inverse): the span-2 twiddle W_4^1.
template <typename R, bool INV>
__device__ __forceinline__ cplx<R> mul_mi(cplx<R> a) {
  return INV ? mk<R>(-a.y, a.x) : mk<R>(a.y, -a.x);
}

// One DIF shuffle stage of span S: lower lane v + p, upper lane (p - v) W_{2S}^{lane mod S}.
template <typename R, int N, bool INV, int S>
__device__ __forceinline__ void dif_shfl(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  constexpr int E = N / 32;
  const bool upper = (lane & S) != 0;
  const R sg = upper ? R(-1) : R(1);
  cplx<R> w = mk<R>(1, 0);
  if (S > 2) w = upper ? twid<R, INV>(tw + tw_off(N, N / (2 * S)), lane & (S - 1)) : mk<R>(1, 0);
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const cplx<R> p = shfl_xor_c<R>(v[j], S);
    cplx<R> t = mk<R>(p.x + sg * v[j].x, p.y + sg * v[j].y);
    if (S == 2) { if (upper && (lane & 1)) t = mul_mi<R, INV>(t); }
    else if (S > 2) t = cmul(t, w);
    v[j] = t;
  }
}

// One DIT shuffle stage of span S: lower lane v + p W, upper lane p - v W (W = W_{2S}^{lane mod S}).
template <typename R, int N, bool INV, int S>
__device__ __forceinline__ void dit_shfl(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  constexpr int E = N / 32;
  const bool upper = (lane & S) != 0;
  const R sg = upper ? R(-1) : R(1);
  cplx<R> w = mk<R>(1, 0);
  if (S > 2) w = twid<R, INV>(tw + tw_off(N, N / (2 * S)), lane & (S - 1));
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const cplx<R> p = shfl_xor_c<R>(v[j], S);
    cplx<R> q = upper ? v[j] : p;          // the operand that carries the twiddle
    const cplx<R> r = upper ? p : v[j];
    if (S == 2) { if (lane & 1) q = mul_mi<R, INV>(q); }
    else if (S > 2) q = cmul(q, w);
    v[j] = mk<R>(r.x + sg * q.x, r.y + sg * q.y);
  }
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
        const int idx = lane + 32 * (j & (half - 1));   // tw[idx * stride]
        v[j + half] = cmul(csub(a, b), twid<R, INV>(tw + tw_off(N, stride), idx));
      }
    }
  }
  // shuffle stages: span 16 ... 1
  dif_shfl<R, N, INV, 16>(v, tw, lane);
  dif_shfl<R, N, INV, 8>(v, tw, lane);
  dif_shfl<R, N, INV, 4>(v, tw, lane);
  dif_shfl<R, N, INV, 2>(v, tw, lane);
  dif_shfl<R, N, INV, 1>(v, tw, lane);
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dit(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  constexpr int E = N / 32;
  constexpr int LE = Log2E<N>::v;
  dit_shfl<R, N, INV, 1>(v, tw, lane);
  dit_shfl<R, N, INV, 2>(v, tw, lane);
  dit_shfl<R, N, INV, 4>(v, tw, lane);
  dit_shfl<R, N, INV, 8>(v, tw, lane);
  dit_shfl<R, N, INV, 16>(v, tw, lane);
#pragma unroll
  for (int m = 0; m < LE; ++m) {
    const int half = 1 << m;
    const int s = 32 * half;
    const int stride = N / (2 * s);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if ((j & half) == 0) {
        const int idx = lane + 32 * (j & (half - 1));   // tw[idx * stride]
        cplx<R> b = cmul(v[j + half], twid<R, INV>(tw + tw_off(N, stride), idx));
        cplx<R> a = v[j];
        v[j] = cadd(a, b);
        v[j + half] = csub(a, b);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Two independent transforms in lockstep (same direction and order): every
// stage issues both arrays' shuffles before their arithmetic, so one warp
// keeps twice the independent work in flight (the kernels are latency bound).
// ---------------------------------------------------------------------------
template <typename R, int N, bool INV, int S>
__device__ __forceinline__ void dif_shfl2(cplx<R> (&a)[N / 32], cplx<R> (&b)[N / 32], const cplx<R>* __restrict__ tw,
                                          int lane) {
  constexpr int E = N / 32;
  const bool upper = (lane & S) != 0;
  const R sg = upper ? R(-1) : R(1);
  cplx<R> w = mk<R>(1, 0);
  if (S > 2) w = upper ? twid<R, INV>(tw + tw_off(N, N / (2 * S)), lane & (S - 1)) : mk<R>(1, 0);
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const cplx<R> pa = shfl_xor_c<R>(a[j], S);
    const cplx<R> pb = shfl_xor_c<R>(b[j], S);
    cplx<R> ta = mk<R>(pa.x + sg * a[j].x, pa.y + sg * a[j].y);
    cplx<R> tb = mk<R>(pb.x + sg * b[j].x, pb.y + sg * b[j].y);
    if (S == 2) {
      if (upper && (lane & 1)) { ta = mul_mi<R, INV>(ta); tb = mul_mi<R, INV>(tb); }
    } else if (S > 2) {
      ta = cmul(ta, w); tb = cmul(tb, w);
    }
    a[j] = ta; b[j] = tb;
  }
}

template <typename R, int N, bool INV, int S>
__device__ __forceinline__ void dit_shfl2(cplx<R> (&a)[N / 32], cplx<R> (&b)[N / 32], const cplx<R>* __restrict__ tw,
                                          int lane) {
  constexpr int E = N / 32;
  const bool upper = (lane & S) != 0;
  const R sg = upper ? R(-1) : R(1);
  cplx<R> w = mk<R>(1, 0);
  if (S > 2) w = twid<R, INV>(tw + tw_off(N, N / (2 * S)), lane & (S - 1));
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const cplx<R> pa = shfl_xor_c<R>(a[j], S);
    const cplx<R> pb = shfl_xor_c<R>(b[j], S);
    cplx<R> qa = upper ? a[j] : pa, qb = upper ? b[j] : pb;
    const cplx<R> ra = upper ? pa : a[j], rb = upper ? pb : b[j];
    if (S == 2) {
      if (lane & 1) { qa = mul_mi<R, INV>(qa); qb = mul_mi<R, INV>(qb); }
    } else if (S > 2) {
      qa = cmul(qa, w); qb = cmul(qb, w);
    }
    a[j] = mk<R>(ra.x + sg * qa.x, ra.y + sg * qa.y);
    b[j] = mk<R>(rb.x + sg * qb.x, rb.y + sg * qb.y);
  }
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dif2(cplx<R> (&a)[N / 32], cplx<R> (&b)[N / 32], const cplx<R>* __restrict__ tw,
                                         int lane) {
  constexpr int E = N / 32;
  constexpr int LE = Log2E<N>::v;
#pragma unroll
  for (int m = LE - 1; m >= 0; --m) {
    const int half = 1 << m;
    const int stride = N / (64 * half);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if ((j & half) == 0) {
        const cplx<R> w = twid<R, INV>(tw + tw_off(N, stride), lane + 32 * (j & (half - 1)));
        const cplx<R> a0 = a[j], a1 = a[j + half], b0 = b[j], b1 = b[j + half];
        a[j] = cadd(a0, a1); b[j] = cadd(b0, b1);
        a[j + half] = cmul(csub(a0, a1), w); b[j + half] = cmul(csub(b0, b1), w);
      }
    }
  }
  dif_shfl2<R, N, INV, 16>(a, b, tw, lane);
  dif_shfl2<R, N, INV, 8>(a, b, tw, lane);
  dif_shfl2<R, N, INV, 4>(a, b, tw, lane);
  dif_shfl2<R, N, INV, 2>(a, b, tw, lane);
  dif_shfl2<R, N, INV, 1>(a, b, tw, lane);
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dit2(cplx<R> (&a)[N / 32], cplx<R> (&b)[N / 32], const cplx<R>* __restrict__ tw,
                                         int lane) {
  constexpr int E = N / 32;
  constexpr int LE = Log2E<N>::v;
  dit_shfl2<R, N, INV, 1>(a, b, tw, lane);
  dit_shfl2<R, N, INV, 2>(a, b, tw, lane);
  dit_shfl2<R, N, INV, 4>(a, b, tw, lane);
  dit_shfl2<R, N, INV, 8>(a, b, tw, lane);
  dit_shfl2<R, N, INV, 16>(a, b, tw, lane);
#pragma unroll
  for (int m = 0; m < LE; ++m) {
    const int half = 1 << m;
    const int stride = N / (64 * half);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      if ((j & half) == 0) {
        const cplx<R> w = twid<R, INV>(tw + tw_off(N, stride), lane + 32 * (j & (half - 1)));
        const cplx<R> ba = cmul(a[j + half], w), bb = cmul(b[j + half], w);
        const cplx<R> a0 = a[j], b0 = b[j];
        a[j] = cadd(a0, ba); a[j + half] = csub(a0, ba);
        b[j] = cadd(b0, bb); b[j + half] = csub(b0, bb);
      }
    }
  }
}

// Cooperative expansion of the N/2-entry twiddle table into the tw_smem(N)
// shared entries (sub-tables of strides 1, 2, ..., N/2 back to back).
template <typename R, int N>
__device__ __forceinline__ void load_twiddles(cplx<R>* s_tw, const cplx<R>* __restrict__ g_tw) {
  for (int i = threadIdx.x; i < tw_smem(N); i += blockDim.x) {
    int r = 1, off = 0;
    while (r < N / 2 && i >= off + N / (2 * r)) { off += N / (2 * r); r *= 2; }
    const int src = (i - off) * r;
    s_tw[i] = g_tw[src < N / 2 ? src : 0];
  }
}

}  // namespace ecs
