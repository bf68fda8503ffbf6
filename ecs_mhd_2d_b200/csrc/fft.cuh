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
// N = 128: radix-4/4/4/2 on the digits of the position; after each local
// radix-4 pass over the register index, the register digit is swapped with the
// next lane digit through a per-warp shared-memory buffer (two exchanges with
// bank-conflict-free, XOR-swizzled addresses), and the last lane digit with a
// register digit by a pairwise shuffle swap fused with the radix-2 pass, so
// every butterfly is local.  The transposed sequence (twiddles before
// butterflies, exchanges reversed) is the DIT.  Fewer instructions than five
// shuffle stages and less shared-memory/shuffle traffic.
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
// N = 128 adds the radix-4 table (R4_TW entries) after the strided ones.
constexpr int R4_TW = 128;
__host__ __device__ constexpr int tw_smem(int N) { return N + (N == 128 ? R4_TW : 0); }
__host__ __device__ constexpr int tw_off(int N, int r) { return N - N / r; }
// Per-warp exchange buffers of the N = 128 transforms (two transforms of N
// entries), placed after the tables; fft_smem(N, W) is the whole region of a
// CTA of W warps, which every kernel that calls a transform reserves.
__host__ __device__ constexpr int fft_xbuf(int N) { return N == 128 ? 2 * N : 0; }
__host__ __device__ constexpr int fft_smem(int N, int W) { return tw_smem(N) + W * fft_xbuf(N); }

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
// N = 128: radix-4/4/4/2 with shared-memory digit exchanges.
// Position e = l + 32 j with l = m + 8 i: pass 1 is the length-4 DFT over j
// (twiddles W_128^{l k1}), pass 2 over i after exchange 1 (W_32^{m q1}), pass 3
// over the next lane digit after exchange 2 (W_8^{p r1}), pass 4 the final
// radix-2 after exchange 3.  Output: lane L, register t holds X[k] with
// k = k1 + 4 q1 + 16 r1 + 64 r2, k1 = L >> 3, q1 = (L >> 1) & 3,
// r1 = (L & 1) + 2 (t >> 1), r2 = t & 1.  Exchange 3 (one digit) is a pairwise
// shuffle swap fused with the radix-2 pass (r2_swap_dif / r2_swap_dit).
// Radix-4 table at tw + 128 (tw[k] = W_128^k): [0, 96) W_128^{l k1} at
// (k1-1)*32 + l; [96, 120) W_32^{m q1} at 96 + (q1-1)*8 + m; [120, 128)
// W_8^{p r1} at 120 + 4p + r1.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int spec128(int lane, int t) {
  return (lane >> 3) + 4 * ((lane >> 1) & 3) + 16 * ((lane & 1) + 2 * (t >> 1)) + 64 * (t & 1);
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

// exchange address maps (entry index in a 128-entry buffer) for lane, register r
__device__ __forceinline__ int x1_w(int lane, int r) { return r * 32 + lane; }
__device__ __forceinline__ int x1_r(int lane, int r) { return (lane >> 3) * 32 + (lane & 7) + 8 * r; }
__device__ __forceinline__ int x2_w(int lane, int r) { return (lane >> 3) * 32 + r * 8 + ((lane & 7) ^ (2 * r)); }
__device__ __forceinline__ int x2_r(int lane, int r) {
  const int p = lane & 1, q1 = (lane >> 1) & 3;
  return (lane >> 3) * 32 + q1 * 8 + ((2 * r + p) ^ (2 * q1));
}

template <typename R, int NT, int WF(int, int), int RF(int, int)>
__device__ __forceinline__ void r4_xchg(cplx<R> (*const (&v)[NT])[4], cplx<R>* xb, int lane) {
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int r = 0; r < 4; ++r) xb[a * 128 + WF(lane, r)] = (*v[a])[r];
  __syncwarp();
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int r = 0; r < 4; ++r) (*v[a])[r] = xb[a * 128 + RF(lane, r)];
  __syncwarp();
}

template <typename R, bool INV>
__device__ __forceinline__ cplx<R> r4_tw(const cplx<R>* t4, int i) {
  cplx<R> w = t4[i];
  if (INV) w.y = -w.y;
  return w;
}

template <typename R, bool INV, int NT>
__device__ __forceinline__ void r4_twiddle(cplx<R> (*const (&v)[NT])[4], const cplx<R>* t4, int base, int stride,
                                           int idx) {
#pragma unroll
  for (int k = 1; k < 4; ++k) {
    const cplx<R> w = r4_tw<R, INV>(t4, base + (k - 1) * stride + idx);
#pragma unroll
    for (int a = 0; a < NT; ++a) (*v[a])[k] = cmul((*v[a])[k], w);
  }
}

template <typename R, bool INV, int NT>
__device__ __forceinline__ void r4_pass(cplx<R> (*const (&v)[NT])[4]) {
#pragma unroll
  for (int a = 0; a < NT; ++a) r4_dft<R, INV>((*v[a])[0], (*v[a])[1], (*v[a])[2], (*v[a])[3]);
}

// The exchange buffer of the calling warp: after the tables, 2 * 128 entries per warp.
template <typename R>
__device__ __forceinline__ cplx<R>* r4_buf(const cplx<R>* tw) {
  return const_cast<cplx<R>*>(tw) + tw_smem(128) + (threadIdx.x >> 5) * fft_xbuf(128);
}

// Exchange 3 fused with the last radix-2 pass: lanes L and L^1 swap the
// register digit r1 & 1 with the lane digit p (each sends one value of each
// register pair), and the pair's butterfly sign follows the lane bit:
// out(r2 = 0) = keep + recv, out(r2 = 1) = (1 - 2b) (keep - recv).
template <typename R, int NT>
__device__ __forceinline__ void r2_swap_dif(cplx<R> (*const (&v)[NT])[4], int lane) {
  const bool b = lane & 1;
  const R sg = b ? R(-1) : R(1);
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int h = 0; h < 4; h += 2) {
      const cplx<R> keep = b ? (*v[a])[h + 1] : (*v[a])[h];
      const cplx<R> send = b ? (*v[a])[h] : (*v[a])[h + 1];
      const cplx<R> recv = shfl_xor_c<R>(send, 1);
      (*v[a])[h] = cadd(keep, recv);
      (*v[a])[h + 1] = cscale(csub(keep, recv), sg);
    }
}

// Transpose of r2_swap_dif: the radix-2 pass, then the lane/register digit swap.
template <typename R, int NT>
__device__ __forceinline__ void r2_swap_dit(cplx<R> (*const (&v)[NT])[4], int lane) {
  const bool b = lane & 1;
  const R sg = b ? R(-1) : R(1);
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int h = 0; h < 4; h += 2) {
      const cplx<R> x = (*v[a])[h], y = cscale((*v[a])[h + 1], sg);
      const cplx<R> keep = cadd(x, y), send = csub(x, y);
      const cplx<R> recv = shfl_xor_c<R>(send, 1);
      (*v[a])[h] = b ? recv : keep;
      (*v[a])[h + 1] = b ? keep : recv;
    }
}

template <typename R, bool INV, int NT>
__device__ __forceinline__ void fft128_dif(cplx<R> (*const (&v)[NT])[4], const cplx<R>* tw, int lane) {
  const cplx<R>* t4 = tw + 128;
  cplx<R>* xb = r4_buf<R>(tw);
  r4_pass<R, INV, NT>(v);
  r4_twiddle<R, INV, NT>(v, t4, 0, 32, lane);
  r4_xchg<R, NT, x1_w, x1_r>(v, xb, lane);
  r4_pass<R, INV, NT>(v);
  r4_twiddle<R, INV, NT>(v, t4, 96, 8, lane & 7);
  r4_xchg<R, NT, x2_w, x2_r>(v, xb, lane);
  r4_pass<R, INV, NT>(v);
  r4_twiddle<R, INV, NT>(v, t4, 121, 1, (lane & 1) * 4);
  r2_swap_dif<R, NT>(v, lane);
}

template <typename R, bool INV, int NT>
__device__ __forceinline__ void fft128_dit(cplx<R> (*const (&v)[NT])[4], const cplx<R>* tw, int lane) {
  const cplx<R>* t4 = tw + 128;
  cplx<R>* xb = r4_buf<R>(tw);
  r2_swap_dit<R, NT>(v, lane);
  r4_twiddle<R, INV, NT>(v, t4, 121, 1, (lane & 1) * 4);
  r4_pass<R, INV, NT>(v);
  r4_xchg<R, NT, x2_r, x2_w>(v, xb, lane);
  r4_twiddle<R, INV, NT>(v, t4, 96, 8, lane & 7);
  r4_pass<R, INV, NT>(v);
  r4_xchg<R, NT, x1_r, x1_w>(v, xb, lane);
  r4_twiddle<R, INV, NT>(v, t4, 0, 32, lane);
  r4_pass<R, INV, NT>(v);
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
  if constexpr (N == 128) {   // radix-4 table: W_128^k with k < 128 from the half table
    for (int i = threadIdx.x; i < R4_TW; i += blockDim.x) {
      int k;
      if (i < 96) k = ((i >> 5) + 1) * (i & 31);
      else if (i < 120) k = 4 * (((i - 96) >> 3) + 1) * ((i - 96) & 7);
      else k = 16 * ((i - 120) >> 2) * ((i - 120) & 3);
      cplx<R> w = g_tw[k & 63];
      if (k & 64) { w.x = -w.x; w.y = -w.y; }
      s_tw[N + i] = w;
    }
  }
}

}  // namespace ecs
