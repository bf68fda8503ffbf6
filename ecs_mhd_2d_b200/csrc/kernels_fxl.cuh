// Tangent (JVP) and adjoint (VJP) of the classic RK4 and Lawson-RK6 shooting
// modes (jax_scripts/lib/timestepping.py:17-44 and :83-125), from one
// description of an explicit (Lawson) Runge-Kutta step:
//
//   x_1 = f0,  k_s = h v(x_s),
//   x_s = e^{p_s} f0 + sum_{j<s} a_sj e^{p_s - p_j} k_j,
//   f'  = e^{P} f0 + sum_j b_j e^{P - p_j} k_j,
//
// where e = exp(tau h L) (masked) is the integrating factor and p_s counts the
// factors applied before stage s.  Lawson-RK6 applies e after stages 1, 3, 4,
// 5, 6 and 7 (p = 0 1 1 2 3 4 5 6, P = 6, tau = 1/6); classic RK4 has no
// factor (e = 1) and its v includes the dissipation L x (loss_functions.py:53).
// The reference repeats the multiplications by e; here powers of e are formed
// by repeated multiplication too, and the stage weights are products with the
// rational coefficients (rounding differences of order 1e-16, far inside the
// parity bound).
//
// With dh = dT / steps, d(e^m) = m tau L e^m dh:
//   dk_s  = (dh/h) k_s + h (N'(x_s) dx_s [+ L dx_s])
//   dx_s  = e^{p_s} (df0 + p_s c f0) + sum_{j<s} a_sj e^{p_s-p_j} (dk_j + (p_s-p_j) c k_j),  c = tau L dh
// and in reverse, from the cotangent fbar' of f':
//   kbar_j = b_j e^{P-p_j} fbar',  f0bar = e^P fbar'
//   for s = S..1:  xbar_s = N'(x_s)^T (h kbar_s) [+ h L kbar_s];
//                  f0bar += e^{p_s} xbar_s,  kbar_j += a_sj e^{p_s-p_j} xbar_s (j < s)
//   hbar = sum_s <kbar_s, k_s>/h + the e^m terms (<ybar, m tau L e^m y>).
#pragma once

#include "kernels_adj.cuh"
#include "kernels_fx.cuh"

namespace ecs {

// Stage count, factor exponent and dissipation-in-v of a scheme.
__host__ __device__ constexpr int fxl_stages(int scheme) { return scheme == FX_RK6 ? 8 : 4; }
__host__ __device__ constexpr double fxl_tau(int scheme) { return scheme == FX_RK6 ? 1.0 / 6.0 : 0.0; }
__host__ __device__ constexpr bool fxl_diss_in_v(int scheme) { return scheme == FX_RK4; }
// p_s (s = 1..S) and P (s = S + 1)
__host__ __device__ constexpr int fxl_p(int scheme, int s) {
  if (scheme != FX_RK6) return 0;
  return s == 1 ? 0 : s <= 3 ? 1 : s <= 8 ? s - 2 : 6;   // 0 1 1 2 3 4 5 6 ; P = 6
}
// a_sj (s = 2..S, j < s); s = S + 1 gives the final weights b_j
__host__ __device__ constexpr double fxl_a(int scheme, int s, int j) {
  if (scheme == FX_RK4) {
    if (s == 5) return j == 1 ? 1.0 / 6.0 : j == 2 ? 1.0 / 3.0 : j == 3 ? 1.0 / 3.0 : 1.0 / 6.0;   // :44
    return (s == 2 && j == 1) ? 0.5 : (s == 3 && j == 2) ? 0.5 : (s == 4 && j == 3) ? 1.0 : 0.0;  // :40-43
  }
  switch (s) {   // timestepping.py:112-124
    case 2: return j == 1 ? 1.0 / 6.0 : 0.0;
    case 3: return (j == 1 || j == 2) ? 1.0 / 12.0 : 0.0;
    case 4: return j == 2 ? -4.0 / 33.0 : j == 3 ? 5.0 / 11.0 : 0.0;
    case 5: return j == 1 ? -1.0 / 4.0 : j == 2 ? -29.0 / 44.0 : j == 3 ? 31.0 / 22.0 : 0.0;
    case 6: return j == 1 ? 3.0 / 11.0 : j == 2 ? 8.0 / 33.0 : j == 3 ? -4.0 / 11.0 : j == 4 ? 1.0 / 11.0
                 : j == 5 ? 14.0 / 33.0 : 0.0;
    case 7: return j == 1 ? -17.0 / 48.0 : j == 2 ? -5.0 / 12.0 : j == 3 ? 1.0 : j == 4 ? 1.0
                 : j == 5 ? -13.0 / 12.0 : j == 6 ? 11.0 / 16.0 : 0.0;
    case 8: return j == 1 ? 20.0 / 39.0 : j == 2 ? 12.0 / 39.0 : j == 3 ? -31.0 / 39.0 : j == 4 ? -1.0 / 39.0
                 : j == 5 ? 34.0 / 39.0 : j == 6 ? -11.0 / 39.0 : j == 7 ? 16.0 / 39.0 : 0.0;
    default:   // 9: final weights
      return (j == 1 || j == 8) ? 13.0 / 200.0 : (j == 3 || j == 7) ? 4.0 / 25.0
           : (j == 4 || j == 6) ? 11.0 / 40.0 : 0.0;
  }
}

// Trajectory record of one step: f0, k_1..k_S (as computed, before any
// factor), the stage inputs x_2..x_S.  2 S box vectors.
__host__ __device__ constexpr int fxr_f() { return 0; }
__host__ __device__ constexpr int fxr_k(int s) { return s; }
__host__ __device__ constexpr int fxr_x(int scheme, int s) { return fxl_stages(scheme) + s - 1; }
__host__ __device__ constexpr int fxr_n(int scheme) { return 2 * fxl_stages(scheme); }

// e^m for a small non-negative m by repeated multiplication (e^0 = 1, also
// where the masked factor is 0).
template <typename R> __device__ __forceinline__ R fxl_pow(R e, int m) {
  R r = R(1);
  for (int i = 0; i < m; ++i) r *= e;
  return r;
}

// ---------------------------------------------------------------------------
// Tangent column pass.  Slots per tangent: df0, dx (the current stage input),
// dk_1..dk_S.  STAGE 0: inverse transforms of df0 (the first stage input).
// STAGE s = 1..S: the forward transform of the tangent row pass at x_s gives
// N'(x_s) dx_s, hence dk_s; then the next stage input dx_{s+1} (or, at s = S,
// the step's result df') and its inverse transforms.
// ---------------------------------------------------------------------------
enum FxtSlot { FT_F = 0, FT_X = 1, FT_K1 = 2 };
__host__ __device__ constexpr int fxt_nslot(int scheme) { return fxl_stages(scheme) + 2; }

template <typename R>
struct ColFxtParams {
  const cplx<R>* H;     // [B][NH][K][N]
  cplx<R>* G;           // [B][NG][K][N]
  cplx<R>* D;           // tangent slots [B][nslot][2][K][M]
  int nslot;
  const cplx<R>* rec;   // this step's record [2S][2][K][M]
  const double* dT;     // [B]
  double h, dscale;     // dh = dT * dscale
  const cplx<R>* tw;
  R nu, eta;
  int B, produce;
};

template <typename R, int N, int SCHEME, int STAGE>
__global__ void __launch_bounds__(128) k_col_fxt(ColFxtParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  constexpr int S = fxl_stages(SCHEME);
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  const int c = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;
  cplx<R>* D = p.D + (size_t)b * p.nslot * VEC;
  const cplx<R>* Q = p.rec;
  const R h = (R)p.h;
  const R dh = (R)(p.dT[b] * p.dscale);
  const R coeff = c == 0 ? p.nu : p.eta;
  cplx<R> r[E];
  if (STAGE > 0) col_load_rhs<R, N>(p.H, b, c, ky, lane, s_tw, r);
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    x[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const size_t o = ((size_t)c * K + ky) * M + slot;
    auto Dq = [&](int q) -> cplx<R>& { return D[q * VEC + o]; };
    auto Qv = [&](int q) -> cplx<R> { return Q[q * VEC + o]; };
    if (STAGE == 0) {
      x[j] = Dq(FT_F);
      continue;
    }
    const R L = diss_L<R>(kx, ky, coeff);   // masked: zero at (0,0)
    const bool msk = !(kx == 0 && ky == 0);
    // the integrating factor of the linearisation's step (as k_fx_setup forms it)
    const R e = SCHEME == FX_RK6 ? (msk ? exp(h / R(6) * L) : R(0)) : R(1);
    const R cf = R(fxl_tau(SCHEME)) * L * dh;   // d(e^m) = m cf e^m
    cplx<R> rv = r[j];                          // N'(x_s) dx_s (no forcing)
    if (fxl_diss_in_v(SCHEME)) rv = cadd(rv, cscale(STAGE == 1 ? Dq(FT_F) : Dq(FT_X), L));
    const cplx<R> dk = cadd(cscale(Qv(fxr_k(STAGE)), dh / h), cscale(rv, h));
    Dq(FT_K1 + STAGE - 1) = dk;
    constexpr int sn = STAGE + 1;               // S + 1: the step's result
    constexpr int pn = fxl_p(SCHEME, sn);
    cplx<R> acc = cscale(cadd(Dq(FT_F), cscale(Qv(fxr_f()), R(pn) * cf)), fxl_pow(e, pn));
#pragma unroll
    for (int jj = 1; jj <= STAGE; ++jj) {
      const double a = fxl_a(SCHEME, sn, jj);
      if (a == 0.0) continue;
      const int m = pn - fxl_p(SCHEME, jj);
      const cplx<R> dkj = jj == STAGE ? dk : Dq(FT_K1 + jj - 1);
      acc = cadd(acc, cscale(cadd(dkj, cscale(Qv(fxr_k(jj)), R(m) * cf)), R(a) * fxl_pow(e, m)));
    }
    if (STAGE < S) Dq(FT_X) = acc;
    else Dq(FT_F) = acc;
    x[j] = acc;
  }
  if (!p.produce) return;
  col_inverse_uv<R, N>(x, p.G, b, c, ky, lane, s_tw);
}

// ---------------------------------------------------------------------------
// Adjoint column pass.  Slots per cotangent: f0bar (FA_F; on entry to a step's
// reverse sweep the cotangent of the step's result f'), kbar_1..kbar_S.
// STAGE S + 1 (seed): kbar_j = b_j e^{P-p_j} f'bar, f0bar = e^P f'bar, and the
// emission of lambda_S = h kbar_S.  STAGE s = S..1: the forward transforms of
// the adjoint row pass at x_s give N'(x_s)^T (h kbar_s), hence xbar_s, which is
// distributed to f0bar and kbar_j (j < s); then lambda_{s-1} is emitted
// (nothing after s = 1).  hbar is accumulated per (b, ky, channel) in hacc.
// ---------------------------------------------------------------------------
enum FxaSlot { FA_F = 0, FA_K1 = 1 };
__host__ __device__ constexpr int fxa_nslot(int scheme) { return fxl_stages(scheme) + 1; }

template <typename R>
struct ColFxaParams {
  const cplx<R>* H;     // [B][NHA][K][N]
  cplx<R>* G;           // [B][NG][K][N] (fields 0..2 written)
  cplx<R>* J;           // adjoint slots [B][nslot][2][K][M]
  int nslot;
  const cplx<R>* rec;   // this step's record [2S][2][K][M]
  double* hacc;         // [B][K][2]
  double h;
  const cplx<R>* tw;
  R nu, eta;
  int B;
};

template <typename R, int N, int SCHEME, int STAGE>
__global__ void __launch_bounds__(128) k_col_fxa(ColFxaParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  constexpr int S = fxl_stages(SCHEME);
  constexpr bool SEED = STAGE == S + 1;
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  const int c = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;
  cplx<R>* J = p.J + (size_t)b * p.nslot * VEC;
  const cplx<R>* Q = p.rec;
  const R h = (R)p.h;
  const R coeff = c == 0 ? p.nu : p.eta;
  const R cky = ky == 0 ? R(1) : R(2);
  cplx<R> xa[E];
  if (!SEED) col_adj_xb<R, N>(p.H, b, c, ky, lane, s_tw, xa);
  double hpart = 0.0;
  cplx<R> lam[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    lam[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const size_t o = ((size_t)c * K + ky) * M + slot;
    const R L = diss_L<R>(kx, ky, coeff);
    const bool msk = !(kx == 0 && ky == 0);
    const R e = SCHEME == FX_RK6 ? (msk ? exp(h / R(6) * L) : R(0)) : R(1);
    const R tl = R(fxl_tau(SCHEME)) * L;        // d(e^m)/dh = m tl e^m
    auto Jq = [&](int q) -> cplx<R>& { return J[q * VEC + o]; };
    auto Qv = [&](int q) -> cplx<R> { return Q[q * VEC + o]; };
    auto ip = [&](cplx<R> a, cplx<R> bb) { return (double)a.x * (double)bb.x + (double)a.y * (double)bb.y; };
    cplx<R> kb = mk<R>(0, 0);   // the kbar whose h-multiple feeds the next adjoint row pass
    if (SEED) {
      constexpr int P = fxl_p(SCHEME, S + 1);
      const cplx<R> fb = Jq(FA_F);
      const R eP = fxl_pow(e, P);
      Jq(FA_F) = cscale(fb, eP);
      if (P > 0) hpart += ip(fb, cscale(Qv(fxr_f()), R(P) * tl * eP));
#pragma unroll
      for (int jj = 1; jj <= S; ++jj) {
        const double bw = fxl_a(SCHEME, S + 1, jj);
        const int m = P - fxl_p(SCHEME, jj);
        const R em = fxl_pow(e, m);
        Jq(FA_K1 + jj - 1) = cscale(fb, R(bw) * em);
        if (bw != 0.0 && m > 0) hpart += ip(fb, cscale(Qv(fxr_k(jj)), R(bw) * R(m) * tl * em));
      }
      kb = Jq(FA_K1 + S - 1);
    } else {
      constexpr int ps = fxl_p(SCHEME, STAGE);
      const cplx<R> ks = Jq(FA_K1 + STAGE - 1);   // kbar_s, complete
      hpart += ip(ks, Qv(fxr_k(STAGE))) / (double)h;
      cplx<R> xb = xa[j];
      if (fxl_diss_in_v(SCHEME)) xb = cadd(xb, cscale(ks, h * L));
      const R eps = fxl_pow(e, ps);
      Jq(FA_F) = cadd(Jq(FA_F), cscale(xb, eps));
      if (ps > 0) hpart += ip(xb, cscale(Qv(fxr_f()), R(ps) * tl * eps));
#pragma unroll
      for (int jj = 1; jj < STAGE; ++jj) {
        const double a = fxl_a(SCHEME, STAGE, jj);
        if (a == 0.0) continue;
        const int m = ps - fxl_p(SCHEME, jj);
        const R em = fxl_pow(e, m);
        Jq(FA_K1 + jj - 1) = cadd(Jq(FA_K1 + jj - 1), cscale(xb, R(a) * em));
        if (m > 0) hpart += ip(xb, cscale(Qv(fxr_k(jj)), R(a) * R(m) * tl * em));
      }
      if (STAGE > 1) kb = Jq(FA_K1 + STAGE - 2);
    }
    lam[j] = cdiv_r(cscale(kb, h), cky);
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) hpart += __shfl_xor_sync(0xffffffffu, hpart, off);
  if (lane == 0) p.hacc[((size_t)b * K + ky) * 2 + c] += hpart;
  if (STAGE == 1) return;
  col_adj_emit<R, N>(lam, p.G, b, c, ky, lane, s_tw);
}

}  // namespace ecs
