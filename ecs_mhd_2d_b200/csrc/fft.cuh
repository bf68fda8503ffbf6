// Warp-level FFTs of length N in {64, 128, 256} (one transform per warp).
//
// Data distribution: lane l holds E = N/32 complex values v[j] at "positions"
// e = l + 32*j.
//
//  * fft_dif : natural-order input  -> permuted output (lane l, register j holds X[spec_pos<N>(l, j)])
//  * fft_dit : permuted input       -> natural-order output
//
// Both are unnormalised.  FWD uses exp(-2 pi i k/N), INV uses exp(+2 pi i k/N).
//
// Algorithm.  One radix-E pass over the register digits (the length-E DFT over
// j, then the twiddles W_N^{l k1}), after which every register digit is a
// finished frequency digit and the remaining 32-point DFTs run over the lane
// digits.  Those are five "half-swap" radix-2 stages: stage t (lane bit t, span
// S = 2^t) swaps lane bit t with a finished register bit rb -- the lane whose
// bit t is c keeps the values whose register bit rb is c and sends the other
// half to lane ^ S -- so that the butterfly over bit t becomes register-local,
// with its sign taken from c:
//   lower = keep + recv,  upper = (1 - 2c) (keep - recv) W_{2S}^{l mod S}.
// Each lane sends E/2 values per stage (a plain shuffle butterfly sends all E),
// and no shared memory is used beyond the tables.  The DIT is the transposed
// sequence (each stage's butterfly transposed and swapped back, then the
// twiddles and the radix-E DFT).  The stage order (t, rb) and the resulting
// output permutation spec_pos are listed below for each N.
//
// Twiddles come from a table tw[k] = exp(-2 pi i k / N), k in [0, N/2),
// computed on the host in long double, and expanded on the host (twiddle_image)
// into the shared-memory layout: one contiguous sub-table per index stride
// r = 1, 2, 4, ...:
//   s_tw[tw_off(N, r) + i] = tw[i r],  i < N / (2 r),  tw_off(N, r) = N - N / r,
// so that the lanes of a stage read consecutive entries, followed by the
// radix-E pass's table s_tw[N + (k1-1)*32 + l] = W_N^{l k1}, k1 = 1..E-1.
#pragma once

#include "common.cuh"

namespace ecs {

__host__ __device__ constexpr int tw_first(int N) { return (N / 32 - 1) * 32; }
// Shared-memory twiddle entries and the offset of the stride-r sub-table.
__host__ __device__ constexpr int tw_smem(int N) { return N + tw_first(N); }
__host__ __device__ constexpr int tw_off(int N, int r) { return N - N / r; }
// Shared-memory region of the transforms of a CTA of W warps (the tables: the
// transforms need no per-warp buffers), which every kernel that calls a
// transform reserves at its start.
__host__ __device__ constexpr int fft_smem(int N, int /*warps*/) { return tw_smem(N); }

template <typename R, bool INV>
__device__ __forceinline__ cplx<R> twid(const cplx<R>* __restrict__ tw, int idx) {
  cplx<R> w = tw[idx];
  if (INV) w.y = -w.y;
  return w;
}

// Multiply by -i (forward) or +i (inverse): W_4^1.
template <typename R, bool INV>
__device__ __forceinline__ cplx<R> mul_mi(cplx<R> a) {
  return INV ? mk<R>(-a.y, a.x) : mk<R>(a.y, -a.x);
}

// Multiply by W_8^1 = (1 -+ i) / sqrt(2).
template <typename R, bool INV>
__device__ __forceinline__ cplx<R> mul_w8(cplx<R> a) {
  const R c = R(0.70710678118654752440084436210484904);
  // products rounded on their own (no contraction with the following sums)
  return INV ? mk<R>(mul_rn(a.x - a.y, c), mul_rn(a.x + a.y, c)) : mk<R>(mul_rn(a.x + a.y, c), mul_rn(a.y - a.x, c));
}

// ---------------------------------------------------------------------------
// Output permutation: lane L, register t holds X[spec_pos<N>(L, t)] (Li, ti
// are the bits of L and t).
//   N =  64: stages (t, rb) = (4,0) (3,0) (2,0) (1,0) (0,0);
//            k = L4 + 2 L3 + 4 L2 + 8 L1 + 16 L0 + 32 t0
//   N = 128: stages (4,0) (3,1) (2,0) (1,1) (0,0);
//            k = k1 + 4 k2, k1 = L4 + 2 L3, k2 = L2 + 2 L1 + 4 L0 + 8 t1 + 16 t0
//   N = 256: stages (4,0) (3,1) (2,2) (1,0) (0,1);
//            k = k1 + 8 k2, k1 = L4 + 2 L3 + 4 L2, k2 = L1 + 2 L0 + 4 t2 + 8 t0 + 16 t1
// ---------------------------------------------------------------------------
template <int N> __host__ __device__ __forceinline__ int spec_pos(int L, int t) {
  auto b = [](int x, int i) { return (x >> i) & 1; };
  if constexpr (N == 64) {
    return b(L, 4) + 2 * b(L, 3) + 4 * b(L, 2) + 8 * b(L, 1) + 16 * b(L, 0) + 32 * b(t, 0);
  } else if constexpr (N == 128) {
    return b(L, 4) + 2 * b(L, 3) + 4 * (b(L, 2) + 2 * b(L, 1) + 4 * b(L, 0) + 8 * b(t, 1) + 16 * b(t, 0));
  } else {
    return b(L, 4) + 2 * b(L, 3) + 4 * b(L, 2) + 8 * (b(L, 1) + 2 * b(L, 0) + 4 * b(t, 2) + 8 * b(t, 0) + 16 * b(t, 1));
  }
}

// Stage list: register bit swapped out at lane bit t.
template <int N, int T> struct StageRB {
  static constexpr int v = N == 64 ? 0 : N == 128 ? ((T == 3 || T == 1) ? 1 : 0)
                                                   : (T == 4 ? 0 : T == 3 ? 1 : T == 2 ? 2 : T == 1 ? 0 : 1);
};

// Length-E DFT over the register index, natural order in and out.
template <typename R, bool INV>
__device__ __forceinline__ void dft4(cplx<R>& a0, cplx<R>& a1, cplx<R>& a2, cplx<R>& a3) {
  const cplx<R> s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = mul_mi<R, INV>(csub(a1, a3));
  a0 = cadd(s02, s13); a1 = cadd(d02, d13); a2 = csub(s02, s13); a3 = csub(d02, d13);
}

template <typename R, bool INV, int E>
__device__ __forceinline__ void dft_reg(cplx<R> (&x)[E]) {
  if constexpr (E == 2) {
    const cplx<R> a = x[0], b = x[1];
    x[0] = cadd(a, b); x[1] = csub(a, b);
  } else if constexpr (E == 4) {
    dft4<R, INV>(x[0], x[1], x[2], x[3]);
  } else {
    // radix-2 split: a_j = x_j + x_{j+4} (even outputs), b_j = (x_j - x_{j+4}) W_8^j (odd outputs)
    cplx<R> a0 = cadd(x[0], x[4]), a1 = cadd(x[1], x[5]), a2 = cadd(x[2], x[6]), a3 = cadd(x[3], x[7]);
    cplx<R> b0 = csub(x[0], x[4]);
    cplx<R> b1 = mul_w8<R, INV>(csub(x[1], x[5]));
    cplx<R> b2 = mul_mi<R, INV>(csub(x[2], x[6]));
    cplx<R> b3 = mul_mi<R, INV>(mul_w8<R, INV>(csub(x[3], x[7])));
    dft4<R, INV>(a0, a1, a2, a3);
    dft4<R, INV>(b0, b1, b2, b3);
    x[0] = a0; x[2] = a1; x[4] = a2; x[6] = a3;
    x[1] = b0; x[3] = b1; x[5] = b2; x[7] = b3;
  }
}

// The radix-E pass (DIF order: DFT, then W_N^{l k1}) and its transpose.
template <typename R, bool INV, int NT, int N, bool TRANSPOSED>
__device__ __forceinline__ void first_pass(cplx<R> (*const (&v)[NT])[N / 32], const cplx<R>* tw, int lane) {
  constexpr int E = N / 32;
  const cplx<R>* t1 = tw + N;
  if constexpr (!TRANSPOSED) {
#pragma unroll
    for (int a = 0; a < NT; ++a) dft_reg<R, INV, E>(*v[a]);
  }
#pragma unroll
  for (int k = 1; k < E; ++k) {
    const cplx<R> w = twid<R, INV>(t1, (k - 1) * 32 + lane);
#pragma unroll
    for (int a = 0; a < NT; ++a) (*v[a])[k] = cmul((*v[a])[k], w);
  }
  if constexpr (TRANSPOSED) {
#pragma unroll
    for (int a = 0; a < NT; ++a) dft_reg<R, INV, E>(*v[a]);
  }
}

// (1 - 2c) W_{2S}^{lane mod S} of a half-swap stage (W = 1 for S = 1; for
// S = 2 only the sign, the W_4 factor is applied as a swap).
template <typename R, bool INV, int N, int S>
__device__ __forceinline__ cplx<R> hs_factor(const cplx<R>* tw, int lane, R sg) {
  if constexpr (S > 2) {
    const cplx<R> w = twid<R, INV>(tw + tw_off(N, N / (2 * S)), lane & (S - 1));
    return mk<R>(sg * w.x, sg * w.y);
  } else {
    return mk<R>(sg, R(0));
  }
}

template <typename R, bool INV, int NT, int N, int T>
__device__ __forceinline__ void hs_dif(cplx<R> (*const (&v)[NT])[N / 32], const cplx<R>* tw, int lane) {
  constexpr int E = N / 32, S = 1 << T, RB = StageRB<N, T>::v;
  const bool c = (lane >> T) & 1;
  const cplx<R> f = hs_factor<R, INV, N, S>(tw, lane, c ? R(-1) : R(1));
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int og = 0; og < E / 2; ++og) {
      const int r0 = (og & ((1 << RB) - 1)) | ((og >> RB) << (RB + 1)), r1 = r0 | (1 << RB);
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

template <typename R, bool INV, int NT, int N, int T>
__device__ __forceinline__ void hs_dit(cplx<R> (*const (&v)[NT])[N / 32], const cplx<R>* tw, int lane) {
  constexpr int E = N / 32, S = 1 << T, RB = StageRB<N, T>::v;
  const bool c = (lane >> T) & 1;
  const cplx<R> f = hs_factor<R, INV, N, S>(tw, lane, c ? R(-1) : R(1));
#pragma unroll
  for (int a = 0; a < NT; ++a)
#pragma unroll
    for (int og = 0; og < E / 2; ++og) {
      const int r0 = (og & ((1 << RB) - 1)) | ((og >> RB) << (RB + 1)), r1 = r0 | (1 << RB);
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

template <typename R, bool INV, int NT, int N>
__device__ __forceinline__ void fft_dif_n(cplx<R> (*const (&v)[NT])[N / 32], const cplx<R>* tw, int lane) {
  first_pass<R, INV, NT, N, false>(v, tw, lane);
  hs_dif<R, INV, NT, N, 4>(v, tw, lane);
  hs_dif<R, INV, NT, N, 3>(v, tw, lane);
  hs_dif<R, INV, NT, N, 2>(v, tw, lane);
  hs_dif<R, INV, NT, N, 1>(v, tw, lane);
  hs_dif<R, INV, NT, N, 0>(v, tw, lane);
}

template <typename R, bool INV, int NT, int N>
__device__ __forceinline__ void fft_dit_n(cplx<R> (*const (&v)[NT])[N / 32], const cplx<R>* tw, int lane) {
  hs_dit<R, INV, NT, N, 0>(v, tw, lane);
  hs_dit<R, INV, NT, N, 1>(v, tw, lane);
  hs_dit<R, INV, NT, N, 2>(v, tw, lane);
  hs_dit<R, INV, NT, N, 3>(v, tw, lane);
  hs_dit<R, INV, NT, N, 4>(v, tw, lane);
  first_pass<R, INV, NT, N, true>(v, tw, lane);
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dif(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  cplx<R>(*const ptrs[1])[N / 32] = {&v};
  fft_dif_n<R, INV, 1, N>(ptrs, tw, lane);
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dit(cplx<R> (&v)[N / 32], const cplx<R>* __restrict__ tw, int lane) {
  cplx<R>(*const ptrs[1])[N / 32] = {&v};
  fft_dit_n<R, INV, 1, N>(ptrs, tw, lane);
}

// Two independent transforms in lockstep (same direction and order): every
// stage issues both arrays' shuffles before their arithmetic, so one warp
// keeps twice the independent work in flight.
template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dif2(cplx<R> (&a)[N / 32], cplx<R> (&b)[N / 32], const cplx<R>* __restrict__ tw,
                                         int lane) {
  cplx<R>(*const ptrs[2])[N / 32] = {&a, &b};
  fft_dif_n<R, INV, 2, N>(ptrs, tw, lane);
}

template <typename R, int N, bool INV>
__device__ __forceinline__ void fft_dit2(cplx<R> (&a)[N / 32], cplx<R> (&b)[N / 32], const cplx<R>* __restrict__ tw,
                                         int lane) {
  cplx<R>(*const ptrs[2])[N / 32] = {&a, &b};
  fft_dit_n<R, INV, 2, N>(ptrs, tw, lane);
}

// The shared-memory twiddle image (tw_smem(N) entries) built from the half
// table half[k] = exp(-2 pi i k / N), k < N/2: the strided sub-tables, then the
// radix-E pass's table W_N^{l k1} (k >= N/2 taken as -W_N^{k - N/2}).  Built
// once on the host when a context is created.
template <typename C, int N>
__host__ __device__ inline void twiddle_image(const C* half, C* img) {
  for (int i = 0; i < N; ++i) {
    int r = 1, off = 0;
    while (r < N / 2 && i >= off + N / (2 * r)) { off += N / (2 * r); r *= 2; }
    const int src = (i - off) * r;
    img[i] = half[src < N / 2 ? src : 0];
  }
  for (int i = 0; i < tw_first(N); ++i) {
    const int k = ((i >> 5) + 1) * (i & 31);
    C w = half[k & (N / 2 - 1)];
    if (k & (N / 2)) { w.x = -w.x; w.y = -w.y; }
    img[N + i] = w;
  }
}

// Copy of the twiddle image into shared memory (cp.async: global -> shared
// without a register round trip); each thread waits for its own copies and the
// caller's __syncthreads makes the table visible.
template <typename R, int N>
__device__ __forceinline__ void load_twiddles(cplx<R>* s_tw, const cplx<R>* __restrict__ g_img) {
  for (int i = threadIdx.x; i < tw_smem(N); i += blockDim.x) cp_async_c<R>(s_tw + i, g_img + i);
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

}  // namespace ecs
