// Warp-level FFTs of length N in {64, 128, 256} (one transform per warp).
//
// Data distribution: lane l holds E = N/32 complex values v[j] at "positions"
// e = l + 32*j.
//
//  * fft_dif : natural-order input  -> permuted output (lane l, register j holds X[spec_pos<N>(l, j)])
//  * fft_dit : permuted input       -> natural-order output
//
// N = 64, 256: radix-2; stages whose butterfly span is >= 32 are
// register-local, the five stages with span < 32 exchange values with
// __shfl_xor_sync; spec_pos(l, j) = bitrev(l + 32 j).
// N = 128: a radix-4 pass over the two register digits, then five radix-2
// stages in which a lane digit is swapped with a finished register digit by
// pairwise shuffles (each lane sends half of its values) and the butterfly is
// local, with its sign taken from the lane bit; half the shuffle traffic of
// the plain radix-2 stages.  The transposed sequence is the DIT.
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
// N = 128 adds the radix-4 pass's table (R4_TW entries) after the strided ones.
constexpr int R4_TW = 96;
__host__ __device__ constexpr int tw_smem(int N) { return N + (N == 128 ? R4_TW : 0); }
__host__ __device__ constexpr int tw_off(int N, int r) { return N - N / r; }
// Shared-memory region of the transforms of a CTA of W warps (the tables; the
// transforms need no per-warp buffers), which every kernel that calls a
// transform reserves at its start.
__host__ __device__ constexpr int fft_smem(int N, int /*warps*/) { return tw_smem(N); }

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

// ---------------------------------------------------------------------------
// N = 128: one radix-4 pass over the register digits, then five half-swap
// radix-2 stages over the lane digits.
// Position e = l + 32 j.  The radix-4 pass is the length-4 DFT over j with the
// twiddles W_128^{l k1} (table at tw + 128, entry (k1-1)*32 + l, k1 = 1..3).
// Stage t (lane bit t, span S = 2^t) swaps lane bit t with a finished register
// bit rb: the lane whose bit t is c keeps its two values whose register bit rb
// is c and sends the other two to lane ^ S (8 32-bit shuffles), and the
// butterfly over the new register bit is local, with its sign taken from c:
// lower = keep + recv, upper = (1 - 2c)(keep - recv) W_{2S}^{l mod S}.  Stages
// (t, rb) = (4,0) (3,1) (2,0) (1,1) (0,0).  Output: lane L, register t holds
// X[k1 + 4 k2] with k1 = L4 + 2 L3, k2 = L2 + 2 L1 + 4 L0 + 8 t1 + 16 t0 (Li,
// ti the bits of L and t).  The DIT is the transposed sequence.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int spec128(int lane, int t) {
  const int k1 = ((lane >> 4) & 1) + 2 * ((lane >> 3) & 1);
  const int k2 = ((lane >> 2) & 1) + 2 * ((lane >> 1) & 1) + 4 * (lane & 1) + 8 * ((t >> 1) & 1) + 16 * (t & 1);
  return k1 + 4 * k2;
}

template <int N> __device__ __forceinline__ int spec_pos(int lane, int j) {
  if constexpr (N == 128) return spec128(lane, j);
  else return bitrev<N>(lane + 32 * j);
}

template <typename R, bool INV>
__device__ __forceinline__ void r4_dft(cplx<R>& a0, cplx<R>& a1, cplx<R>& a2, cplx<R>& a3) {
  const cplx<R> s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = mul_mi<R, INV>(csub(a1, a3));
  a0 = cadd(s02, s13); a1 = cadd(d02, d13); a2 = csub(s02, s13); a3 = csub(d02, d13);
}

// The radix-4 pass: DFT over the register index, then W_128^{l k1} on k1 = 1..3.
template <typename R, bool INV, int NT>
__device__ __forceinline__ void r4_first(cplx<R> (*const (&v)[NT])[4], const cplx<R>* t4, int lane) {
#pragma unroll
  for (int a = 0; a < NT; ++a) r4_dft<R, INV>((*v[a])[0], (*v[a])[1], (*v[a])[2], (*v[a])[3]);
#pragma unroll
  for (int k = 1; k < 4; ++k) {
    const cplx<R> w = twid<R, INV>(t4, (k - 1) * 32 + lane);
#pragma unroll
    for (int a = 0; a < NT; ++a) (*v[a])[k] = cmul((*v[a])[k], w);
  }
}

// Transpose of r4_first: the twiddles, then the DFT over the register index.
template <typename R, bool INV, int NT>
__device__ __forceinline__ void r4_last(cplx<R> (*const (&v)[NT])[4], const cplx<R>* t4, int lane) {
#pragma unroll
  for (int k = 1; k < 4; ++k) {
    const cplx<R> w = twid<R, INV>(t4, (k - 1) * 32 + lane);
#pragma unroll
    for (int a = 0; a < NT; ++a) (*v[a])[k] = cmul((*v[a])[k], w);
  }
#pragma unroll
  for (int a = 0; a < NT; ++a) r4_dft<R, INV>((*v[a])[0], (*v[a])[1], (*v[a])[2], (*v[a])[3]);
}

// (1 - 2c) W_{2S}^{lane mod S} for a half-swap stage of span S (W = 1 for S = 1).
template <typename R, bool INV, int S>
__device__ __forceinline__ cplx<R> hs_factor(const cplx<R>* tw, int lane, R sg) {
  if constexpr (S > 2) {
    const cplx<R> w = twid<R, INV>(tw + tw_off(128, 128 / (2 * S)), lane & (S - 1));
    return mk<R>(sg * w.x, sg * w.y);
  } else {
    return mk<R>(sg, R(0));
  }
}

template <typename R, bool INV, int NT, int T, int RB>
__device__ __forceinline__ void hs_dif(cplx<R> (*const (&v)[NT])[4], const cplx<R>* tw, int lane) {
  constexpr int S = 1 << T;
  const bool c = (lane >> T) & 1;
  const cplx<R> f = hs_factor<R, INV, S>(tw, lane, c ? R(-1) : R(1));
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int og = 0; og < 2; ++og) {
      constexpr int o = 1 - RB;
      const int r0 = og << o, r1 = (1 << RB) | (og << o);
      const cplx<R> keep = c ? (*v[a])[r1] : (*v[a])[r0];
      const cplx<R> send = c ? (*v[a])[r0] : (*v[a])[r1];
      const cplx<R> recv = shfl_xor_c<R>(send, S);
      (*v[a])[r0] = cadd(keep, recv);
      cplx<R> d = csub(keep, recv);
      if constexpr (S > 2) d = cmul(d, f);
      else {
        d = cscale(d, f.x);
        if constexpr (S == 2) { if (lane & 1) d = mul_mi<R, INV>(d); }
      }
      (*v[a])[r1] = d;
    }
}

template <typename R, bool INV, int NT, int T, int RB>
__device__ __forceinline__ void hs_dit(cplx<R> (*const (&v)[NT])[4], const cplx<R>* tw, int lane) {
  constexpr int S = 1 << T;
  const bool c = (lane >> T) & 1;
  const cplx<R> f = hs_factor<R, INV, S>(tw, lane, c ? R(-1) : R(1));
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int og = 0; og < 2; ++og) {
      constexpr int o = 1 - RB;
      const int r0 = og << o, r1 = (1 << RB) | (og << o);
      cplx<R> y = (*v[a])[r1];
      if constexpr (S > 2) y = cmul(y, f);
      else {
        if constexpr (S == 2) { if (lane & 1) y = mul_mi<R, INV>(y); }
        y = cscale(y, f.x);
      }
      const cplx<R> x = (*v[a])[r0];
      const cplx<R> keep = cadd(x, y), send = csub(x, y);
      const cplx<R> recv = shfl_xor_c<R>(send, S);
      (*v[a])[r0] = c ? recv : keep;
      (*v[a])[r1] = c ? keep : recv;
    }
}

template <typename R, bool INV, int NT>
__device__ __forceinline__ void fft128_dif(cplx<R> (*const (&v)[NT])[4], const cplx<R>* tw, int lane) {
  r4_first<R, INV, NT>(v, tw + 128, lane);
  hs_dif<R, INV, NT, 4, 0>(v, tw, lane);
  hs_dif<R, INV, NT, 3, 1>(v, tw, lane);
  hs_dif<R, INV, NT, 2, 0>(v, tw, lane);
  hs_dif<R, INV, NT, 1, 1>(v, tw, lane);
  hs_dif<R, INV, NT, 0, 0>(v, tw, lane);
}

template <typename R, bool INV, int NT>
__device__ __forceinline__ void fft128_dit(cplx<R> (*const (&v)[NT])[4], const cplx<R>* tw, int lane) {
  hs_dit<R, INV, NT, 0, 0>(v, tw, lane);
  hs_dit<R, INV, NT, 1, 1>(v, tw, lane);
  hs_dit<R, INV, NT, 2, 0>(v, tw, lane);
  hs_dit<R, INV, NT, 3, 1>(v, tw, lane);
  hs_dit<R, INV, NT, 4, 0>(v, tw, lane);
  r4_last<R, INV, NT>(v, tw + 128, lane);
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dif(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  if constexpr (N == 128) {
    cplx<R>(*const ptrs[1])[4] = {&v};
    fft128_dif<R, INV, 1>(ptrs, tw, lane);
    return;
  }
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
  if constexpr (N == 128) {
    cplx<R>(*const ptrs[1])[4] = {&v};
    fft128_dit<R, INV, 1>(ptrs, tw, lane);
    return;
  }
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
  if constexpr (N == 128) {
    cplx<R>(*const ptrs[2])[4] = {&a, &b};
    fft128_dif<R, INV, 2>(ptrs, tw, lane);
    return;
  }
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
  if constexpr (N == 128) {
    cplx<R>(*const ptrs[2])[4] = {&a, &b};
    fft128_dit<R, INV, 2>(ptrs, tw, lane);
    return;
  }
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
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    int r = 1, off = 0;
    while (r < N / 2 && i >= off + N / (2 * r)) { off += N / (2 * r); r *= 2; }
    const int src = (i - off) * r;
    s_tw[i] = g_tw[src < N / 2 ? src : 0];
  }
  if constexpr (N == 128) {   // radix-4 table: W_128^{l k1} at (k1-1)*32 + l from the half table
    for (int i = threadIdx.x; i < R4_TW; i += blockDim.x) {
      const int k = ((i >> 5) + 1) * (i & 31);
      cplx<R> w = g_tw[k & 63];
      if (k & 64) { w.x = -w.x; w.y = -w.y; }
      s_tw[N + i] = w;
    }
  }
}

}  // namespace ecs
