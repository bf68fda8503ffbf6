// Common device helpers for the ECS-MHD-2D B200 kernels.
//
// Spectral "box" layout (all hot kernels):
//   The 2/3 dealiasing mask of the reference (jax_scripts/lib/mhd_jax.py:65-70)
//   keeps |kx| < n/3 and |ky| < n/3.  Every hot-path state lives only on those
//   modes, so the state is stored compactly as
//       V[b][c][ky][slot]      c in {omega, j}, ky in [0, K), slot in [0, M)
//   with kmax = (n-1)/3, K = kmax+1, M = 2*kmax+1 and
//       kx(slot) = slot (slot <= kmax),  slot - M (slot > kmax).
//   A column (fixed ky) is contiguous, which is what the column kernels read.
//   FFT position p (fftfreq order, length n) <-> slot: p = kx mod n.
//
// Intermediate layouts (per batch element):
//   G[b][field][ky][x]   column-inverse-transformed fields (complex, x contiguous)
//   H[b][field][ky][x]   row-forward-transformed fields      (complex, x contiguous)
//   Phys[x][field][pos]  physical rows in warp-FFT position order (primal record)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ecs {

template <typename R> struct CplxT;
template <> struct CplxT<double> { using type = double2; };
template <> struct CplxT<float>  { using type = float2; };
template <typename R> using cplx = typename CplxT<R>::type;

template <typename R> __host__ __device__ __forceinline__ cplx<R> mk(R x, R y) { cplx<R> c; c.x = x; c.y = y; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { a.x += b.x; a.y += b.y; return a; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <typename C, typename R> __device__ __forceinline__ C cscale(C a, R s) { a.x *= s; a.y *= s; return a; }
// (i*mu) * z for real mu, written exactly as the reference's `1j * mu * z`.
template <typename C, typename R> __device__ __forceinline__ C cimul(C z, R mu) {
  C r; r.x = -mu * z.y; r.y = mu * z.x; return r;
}
template <typename C, typename R> __device__ __forceinline__ C cdiv_r(C a, R s) { a.x = a.x / s; a.y = a.y / s; return a; }

// x / D for a positive integer constant D, correctly rounded, without a
// division instruction.  A power of two is an exact multiplication.  Otherwise
// (odd part of D at least 3): q0 = x RN(1/D); the residual r = x - q0 D is
// exact in one FMA; q = RN(q0 + r RN(1/D)) is one more FMA (Markstein's
// correction step, P. Markstein, IBM J. Res. Dev. 34(1), 1990).  q is RN(x/D)
// for normal x: q0 + r RN(1/D) differs from x/D by at most ~2^-52 ulp, and x/D
// is never a rounding midpoint (D times a 54-bit odd midpoint significand has
// more than 53 significant bits), being at least ulp/(2D) away from one.  So
// the stepper algebra keeps the operation order and the results of x / D.
template <int D, typename R> __device__ __forceinline__ R div_k(R x) {
  static_assert(D > 0, "positive divisor");
  constexpr R inv = R(1) / R(D);
  if constexpr ((D & (D - 1)) == 0) {
    return x * inv;
  } else {
    const R q0 = x * inv;
    const R r = fma(-q0, R(D), x);
    return fma(r, inv, q0);
  }
}
// a sa + b sb with each product and the sum rounded on their own (never
// contracted into an FMA), so that the same formula compiled into different
// kernels gives the same bits.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
template <typename C, typename R> __device__ __forceinline__ C lin2_rn(C a, R sa, C b, R sb) {
  C r;
  r.x = add_rn(mul_rn(a.x, sa), mul_rn(b.x, sb));
  r.y = add_rn(mul_rn(a.y, sa), mul_rn(b.y, sb));
  return r;
}
template <int D, typename C> __device__ __forceinline__ C cdiv_k(C a) { a.x = div_k<D>(a.x); a.y = div_k<D>(a.y); return a; }
// a b + c d and a b - c d with the rounding fixed: the second product rounded,
// then one FMA.  Written out so that no kernel's compilation chooses another
// contraction: the same formula gives the same bits in every kernel (the
// cluster-resident passes reuse the per-pass kernels' bodies and must agree
// with them bit for bit).
template <typename R> __device__ __forceinline__ R fpp(R a, R b, R c, R d) { return fma(a, b, mul_rn(c, d)); }
template <typename R> __device__ __forceinline__ R fpm(R a, R b, R c, R d) { return fma(a, b, -mul_rn(c, d)); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = fpm(a.x, b.x, a.y, b.y); r.y = fpp(a.x, b.y, a.y, b.x); return r;
}
// s a with each component product rounded on its own (no contraction with a later sum).
template <typename C, typename R> __device__ __forceinline__ C cscale_rn(C a, R s) {
  a.x = mul_rn(a.x, s); a.y = mul_rn(a.y, s); return a;
}
// a + b s, the product rounded on its own.
template <typename C, typename R> __device__ __forceinline__ C cadd_scaled_rn(C a, C b, R s) {
  a.x = add_rn(a.x, mul_rn(b.x, s)); a.y = add_rn(a.y, mul_rn(b.y, s)); return a;
}

template <typename R> __device__ __forceinline__ cplx<R> shfl_xor_c(cplx<R> v, int m) {
  v.x = __shfl_xor_sync(0xffffffffu, v.x, m);
  v.y = __shfl_xor_sync(0xffffffffu, v.y, m);
  return v;
}
// One complex value copied global -> shared with cp.async (no register round
// trip; 16 bytes for double, 8 for float); completed by cp.async.wait_all.
template <typename R> __device__ __forceinline__ void cp_async_c(cplx<R>* dst_smem, const cplx<R>* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  if constexpr (sizeof(cplx<R>) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
// One value of 4, 8 or 16 bytes copied global -> shared with cp.async.
template <typename T> __device__ __forceinline__ void cp_async_v(T* dst_smem, const T* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst_smem);
  if constexpr (sizeof(T) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
template <typename R> __device__ __forceinline__ cplx<R> shfl_c(cplx<R> v, int src) {
  v.x = __shfl_sync(0xffffffffu, v.x, src);
  v.y = __shfl_sync(0xffffffffu, v.y, src);
  return v;
}

// Programmatic dependent launch.  A stepping kernel is launched with
// programmatic stream serialization, so it may start while its predecessor in
// the stream is still running.  It calls pdl_trigger() first (its successor may
// be scheduled once every CTA of this grid has started) and pdl_wait() before
// its first access to global memory other than the constant twiddle table:
// the wait returns when the predecessor grid has completed and its writes are
// visible.  Every such kernel waits before any early return, so completion of
// a grid implies completion of all grids before it.  Both are no-ops for a
// kernel launched without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Box geometry for a grid side n.
struct Geom {
  int n, kmax, K, M;
};
__host__ __device__ inline Geom make_geom(int n) {
  Geom g; g.n = n; g.kmax = (n - 1) / 3; g.K = g.kmax + 1; g.M = 2 * g.kmax + 1; return g;
}
// FFT position -> slot (or -1 when outside the box).
__host__ __device__ __forceinline__ int pos_to_slot(int p, int n, int kmax, int M) {
  if (p <= kmax) return p;
  if (p >= n - kmax) return p - n + M;
  return -1;
}
__host__ __device__ __forceinline__ int slot_to_kx(int s, int kmax, int M) { return s <= kmax ? s : s - M; }
__host__ __device__ __forceinline__ int pos_to_k(int p, int n) { return p <= n / 2 ? p : p - n; }

template <int N> __device__ __forceinline__ int bitrev(int e) {
  constexpr int B = (N == 64) ? 6 : (N == 128) ? 7 : (N == 256) ? 8 : (N == 32) ? 5 : 0;
  static_assert(B > 0, "unsupported N");
  return (int)(__brev((unsigned)e) >> (32 - B));
}

// Per-batch-element control block for the fixed-step and adaptive steppers.
struct StepCtl {
  double t;        // integration time of the call (Lawson-RK43: the horizon T)
  double h;        // current step (Lawson-RK4: (T/nc)/ms)
  double s;        // Lawson-RK43 pseudo-time in [0, 1]
  double err;      // last error estimate (Lawson-RK43)
  int accepted, rejected, fevals, done;
  int pending_accept;   // last attempt accepted, state not yet promoted
  int attempts;         // attempts recorded
  unsigned long long err_bits;  // atomicMax scratch for |err| (non-negative doubles)
  unsigned int err_blocks;      // blocks that have reported their error partial
  int steps_total;              // slot pool: fixed steps of the request
  int steps_done;               // slot pool: steps taken
  int pad;
};

}  // namespace ecs
