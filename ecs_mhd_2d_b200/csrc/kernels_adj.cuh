// Adjoint (reverse-mode) kernels of the shooting map: the VJP used by
// adjoint descent (reference: jax.value_and_grad of loss_RPO,
// jax_scripts/adjoint_descent.py:90-91) and as the transpose preconditioner
// of Newton-GMRES (jax.vjp of objective_RPO, jax_scripts/newton.py:168-170).
//
// Inner products: box vectors use <X, Y> = Re sum conj(X) Y, real fields the
// Euclidean dot.  With these, the transposes of the box transforms are
//   to_box^T(Y)   = n^2 irfft2(Y / c_ky)        (c_ky = 1 for ky = 0, else 2)
//   from_box^T(w) = (c_ky / n^2) rfft2(w)
// so one adjoint right-hand side is again a column pass and a row pass
// (Basdevant form of the products, see kernels.cuh):
//   lambda -> P1bar = Re sum (-kx ky) lambda_w e^{ik.x},  P2bar = Re sum (ky^2 - kx^2) lambda_w e^{ik.x},
//             P3bar = Re sum k^2 lambda_j e^{ik.x}
//   -> product adjoints with the primal fields
//        ubar  =  2u P1bar - v P2bar + B_y P3bar,   vbar  = -2v P1bar - u P2bar - B_x P3bar,
//        Bxbar = -2B_x P1bar + B_y P2bar - v P3bar, Bybar =  2B_y P1bar + B_x P2bar + u P3bar
//   -> 4 forward transforms
//   -> Xbar_c = (c_ky/n^2) sum_m (-i mu_m) rfft2(fbar_mc), mu_m in {ky/k^2, -kx/k^2}.
#pragma once

#include "kernels.cuh"
#include "kernels_rk43.cuh"
#include "kernels_tan.cuh"

namespace ecs {

// ---------------------------------------------------------------------------
// Adjoint row pass
// ---------------------------------------------------------------------------
template <typename R>
struct RowAdjParams {
  const cplx<R>* G;     // [B][NG][K][N]: fields 0..2 hold the inverse columns of the P1, P2, P3 cotangents (/c_ky)
  cplx<R>* H;           // [B][NHA][K][N]: rfft2 rows of the 4 adjoint fields
  const R* phys;        // primal physical fields of this stage: phys + b * phys_bstride is [N][NPH][N]
  long phys_bstride;    // 0: one primal shared by the batch
  const StepCtl* ctl;   // optional per-candidate control: batch elements whose ctl.done is set are skipped
  const cplx<R>* tw;
  int B;
};

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_adj(RowAdjParams<R> p) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_G = s_tw + fft_smem(N, XT);
  cplx<R>* s_H = s_G + 3 * K * (XT + 1);
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = x0 + w;
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  if (p.ctl && p.ctl[b].done) return;   // the whole CTA belongs to batch element b
  const R* ph = phys_row<R, N>(p.phys + (size_t)b * p.phys_bstride, x);
  R pu[E], pv[E], pbx[E], pby[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int e = lane + 32 * j;
    pu[j] = ph[e]; pv[j] = ph[N + e]; pbx[j] = ph[2 * N + e]; pby[j] = ph[3 * N + e];
  }
  load_tile<R, N, XT>(s_G, p.G + (size_t)b * NG * K * N, 3 * K, x0);
  __syncthreads();
  cplx<R> P12[E], P3[E];   // (P1bar, P2bar) and (P3bar, 0) in position order
#pragma unroll
  for (int j = 0; j < E; ++j) {
    P12[j] = packed_pair<R, N, XT>(s_G, s_G + K * (XT + 1), lane + 32 * j, w);
    P3[j] = packed_one<R, N, XT>(s_G + 2 * K * (XT + 1), lane + 32 * j, w);
  }
  fft_dif2<R, N, true>(P12, P3, s_tw, lane);
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const R p1 = P12[j].x, p2 = P12[j].y, p3 = P3[j].x;
    const R u = pu[j], v = pv[j], bx = pbx[j], by = pby[j];
    P12[j] = mk<R>(R(2) * u * p1 - v * p2 + by * p3, -R(2) * v * p1 - u * p2 - bx * p3);     // (ubar, vbar)
    P3[j] = mk<R>(-R(2) * bx * p1 + by * p2 - v * p3, R(2) * by * p1 + bx * p2 + u * p3);    // (Bxbar, Bybar)
  }
  fft_dit2<R, N, false>(P12, P3, s_tw, lane);
  split_store<R, N, XT>(P12, s_H, s_H + K * (XT + 1), w, lane);
  split_store<R, N, XT>(P3, s_H + 2 * K * (XT + 1), s_H + 3 * K * (XT + 1), w, lane);
  __syncthreads();
  store_tile<R, N, XT>(p.H + (size_t)b * NHA * K * N, s_H, NHA * K, x0);
}

// ---------------------------------------------------------------------------
// Adjoint column pass
// ---------------------------------------------------------------------------
enum AdjStage : int {
  AJ_PRE = 0,                        // Lawson-RK4: seed the step adjoint from obar
  AJ_S4 = 4, AJ_S3 = 3, AJ_S2 = 2, AJ_S1 = 1,
  AJ43_INIT = 10,                    // Lawson-RK4(3): adjoint of the initial k1 = t v(x0)
  AJ43_PRE = 11,                     // seed an accepted attempt from (xbar_f, k5bar)
  AJ43_S5 = 15, AJ43_S4 = 14, AJ43_S3 = 13, AJ43_S2 = 12,
  AJ43_IPRE = 16,                    // seed the adjoint RHS of the initial k1
};
// Adjoint slots. Lawson-RK4: OB (obar / fbar), F2, A1, K2, B3.
enum AdjSlot4 { J_OB = 0, J_F2, J_A1, J_K2, J_B3, J_NS4 };
// Lawson-RK4(3): X0 (x0bar carried), K1 (k1bar carried), XF, X2, XB, K1P (k1'bar), K2, K3P (k3'bar), K2P (k2'bar), K1PP
enum AdjSlot43 { JJ_X0 = 0, JJ_K1, JJ_X2, JJ_XB, JJ_K1P, JJ_K1PP, JJ_K2, JJ_K2P, JJ_K3P, JJ_NS43 };

template <typename R>
struct ColAdjParams {
  const cplx<R>* H;     // [B][NHA][K][N]
  cplx<R>* G;           // [B][NG][K][N] (fields 0..2 written)
  cplx<R>* J;           // adjoint slots [B][nslot][2][K][M]
  int nslot;
  const cplx<R>* rec;   // primal record of this step / attempt
  const cplx<R>* rec_prev;   // Lawson-RK4 AJ_S1: record of the previous step (null at the first step)
  double* hacc;         // [B][K][2] accumulators of dL/dh (RK4) or dL/dt (RK4(3))
  double t, h;
  const cplx<R>* tw;
  R nu, eta;
  int B, stage;
  // Several candidates (Lawson-RK4 stages): ctl[b] gives candidate b's step h
  // and done flag (skipped once done); rec / rec_prev + b * rec_bstride its record.
  const StepCtl* ctl;
  long rec_bstride;
};

__device__ __forceinline__ double rdot2(double ax, double ay, double bx, double by) { return ax * bx + ay * by; }

template <typename R, int N, int STAGE>
__global__ void __launch_bounds__(128) k_col_adj(ColAdjParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  const int ch = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;   // one warp per (b, ky, channel)
  if (p.ctl && p.ctl[b].done) return;
  cplx<R>* J = p.J + (size_t)b * p.nslot * VEC;
  const cplx<R>* Q = p.rec + (size_t)b * p.rec_bstride;
  const cplx<R>* Qp = p.rec_prev ? p.rec_prev + (size_t)b * p.rec_bstride : nullptr;
  const R h = p.ctl ? (R)p.ctl[b].h : (R)p.h, t = (R)p.t;
  constexpr bool rk43 = STAGE >= AJ43_INIT;
  constexpr bool has_rhs = !(STAGE == AJ_PRE || STAGE == AJ43_PRE || STAGE == AJ43_IPRE);
  const R cky = ky == 0 ? R(1) : R(2);
  const R inv_n2 = R(1) / (R(N) * R(N));
  const R coeff = ch == 0 ? p.nu : p.eta;

  // Xbar_c = (c_ky/n^2) sum_m (-i mu_m) rfft2(fbar_{m,c}), m over the two uncurled fields of channel c
  cplx<R> xb[E];
#pragma unroll
  for (int j = 0; j < E; ++j) xb[j] = mk<R>(0, 0);
  if (has_rhs) {
    const cplx<R>* h0 = p.H + ((size_t)(b * NHA + 2 * ch) * K + ky) * N;
    const cplx<R>* h1 = h0 + (size_t)K * N;
    cplx<R> v1[E];
#pragma unroll
    for (int j = 0; j < E; ++j) { xb[j] = h0[lane + 32 * j]; v1[j] = h1[lane + 32 * j]; }
    fft_dif2<R, N, false>(xb, v1, s_tw, lane);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      xb[j] = cadd(cimul(xb[j], -spectral_mu<R>(2, kx, ky)), cimul(v1[j], -spectral_mu<R>(3, kx, ky)));
    }
#pragma unroll
    for (int j = 0; j < E; ++j) xb[j] = cscale(xb[j], cky * inv_n2);
  }

  double hpart = 0.0;
  bool feed = true;
  cplx<R> lam[E];   // next adjoint-RHS input lambda / c_ky (multipliers applied per product below)
#pragma unroll
  for (int j = 0; j < E; ++j) {
    lam[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const bool in_mask = !(kx == 0 && ky == 0);
    const size_t o = ((size_t)ch * K + ky) * M + slot;
    const R L = diss_L<R>(kx, ky, coeff);
    const cplx<R> Xb = xb[j];
    cplx<R> kb = mk<R>(0, 0);   // cotangent fed to the next adjoint RHS (before the h or t factor)
    auto ip = [&](cplx<R> a, cplx<R> bb) { return rdot2(a.x, a.y, bb.x, bb.y); };
    if (!rk43) {
      const R e = in_mask ? exp(h / R(2) * L) : R(0);
      const R dedh = e * L / R(2);
      switch (STAGE) {
        case AJ_PRE: {
          const cplx<R> ob = J[J_OB * VEC + o];
          J[J_F2 * VEC + o] = ob; J[J_A1 * VEC + o] = cdiv_k<6>(ob);
          J[J_K2 * VEC + o] = cdiv_k<3>(ob); J[J_B3 * VEC + o] = cdiv_k<3>(ob);
          kb = cdiv_k<6>(ob);                                   // k4bar
          hpart += ip(kb, Q[Q_K4 * VEC + o]) / (double)h;
        } break;
        case AJ_S4: {
          const cplx<R> f2b = cadd(J[J_F2 * VEC + o], Xb), b3b = cadd(J[J_B3 * VEC + o], Xb);
          const cplx<R> b2b = J[J_K2 * VEC + o], b1b = J[J_A1 * VEC + o];
          const cplx<R> f = Q[Q_F * VEC + o], k1 = Q[Q_K1 * VEC + o];
          const double eb = ip(b3b, Q[Q_K3 * VEC + o]) + ip(b2b, Q[Q_K2 * VEC + o]) + ip(b1b, cscale(k1, e)) +
                            ip(f2b, cscale(f, e));
          hpart += eb * (double)dedh;
          kb = cscale(b3b, e);                                     // k3bar
          hpart += ip(kb, Q[Q_K3 * VEC + o]) / (double)h;
          J[J_F2 * VEC + o] = cscale(f2b, e);                      // f1bar
          J[J_A1 * VEC + o] = cscale(b1b, e);                      // a1bar
          J[J_K2 * VEC + o] = cscale(b2b, e);                      // k2bar
        } break;
        case AJ_S3: {
          J[J_F2 * VEC + o] = cadd(J[J_F2 * VEC + o], Xb);
          kb = cadd(J[J_K2 * VEC + o], cscale(Xb, R(0.5)));        // k2bar final
          hpart += ip(kb, Q[Q_K2 * VEC + o]) / (double)h;
        } break;
        case AJ_S2: {
          const cplx<R> f1b = cadd(J[J_F2 * VEC + o], Xb);
          const cplx<R> a1b = cadd(J[J_A1 * VEC + o], cscale(Xb, R(0.5)));
          const double eb = ip(a1b, Q[Q_K1 * VEC + o]) + ip(f1b, Q[Q_F * VEC + o]);
          hpart += eb * (double)dedh;
          kb = cscale(a1b, e);                                     // k1bar
          hpart += ip(kb, Q[Q_K1 * VEC + o]) / (double)h;
          J[J_OB * VEC + o] = cscale(f1b, e);                      // fbar (without the RHS1 term)
        } break;
        default: {   // AJ_S1: fbar += X1bar; then seed the previous step (if any)
          const cplx<R> fb = cadd(J[J_OB * VEC + o], Xb);
          J[J_OB * VEC + o] = fb;
          if (Qp) {
            J[J_F2 * VEC + o] = fb; J[J_A1 * VEC + o] = cdiv_k<6>(fb);
            J[J_K2 * VEC + o] = cdiv_k<3>(fb); J[J_B3 * VEC + o] = cdiv_k<3>(fb);
            kb = cdiv_k<6>(fb);
            hpart += ip(kb, Qp[Q_K4 * VEC + o]) / (double)h;
          } else {
            feed = false;
          }
        } break;
      }
      kb = cscale(kb, h);
    } else {
      const cplx<R> eg = Q[RR_E * VEC + o];   // (e, e L h/2) of the attempt, e = exp(t L h/2)
      const R e = eg.x;
      const R dedt = eg.y;
      switch (STAGE) {
        case AJ43_PRE:      // from (xbar_f, k5bar) in (X0, K1) slots: RHS5 input = k5bar
        case AJ43_IPRE: {   // initial k1 = t v(x0): input = k1bar
          kb = J[JJ_K1 * VEC + o];
          hpart += ip(kb, Q[(STAGE == AJ43_PRE ? RR_K5 : RR_K1) * VEC + o]) / (double)t;
        } break;
        case AJ43_S5: {     // xbar_f += Xbar5; distribute to x2, k1'', k2', k3', k4
          const cplx<R> xfb = cadd(J[JJ_X0 * VEC + o], Xb);
          J[JJ_X2 * VEC + o] = xfb;
          J[JJ_K1PP * VEC + o] = cdiv_k<6>(cscale(xfb, h));
          J[JJ_K2P * VEC + o] = cdiv_k<3>(cscale(xfb, h));
          J[JJ_K3P * VEC + o] = cdiv_k<3>(cscale(xfb, h));
          kb = cdiv_k<6>(cscale(xfb, h));                       // k4bar
          hpart += ip(kb, Q[RR_K4 * VEC + o]) / (double)t;
        } break;
        case AJ43_S4: {     // Y4 = x2 + h k3'
          const cplx<R> x2b = cadd(J[JJ_X2 * VEC + o], Xb);
          const cplx<R> k3pb = cadd(J[JJ_K3P * VEC + o], cscale(Xb, h));
          const cplx<R> k2pb = J[JJ_K2P * VEC + o], k1ppb = J[JJ_K1PP * VEC + o];
          const cplx<R> x0 = Q[RR_X0 * VEC + o], k1 = Q[RR_K1 * VEC + o];
          const double eb = ip(k3pb, Q[RR_K3 * VEC + o]) + ip(k2pb, Q[RR_K2 * VEC + o]) +
                            ip(k1ppb, cscale(k1, e)) + ip(x2b, cscale(x0, e));
          hpart += eb * (double)dedt;
          kb = cscale(k3pb, e);                                    // k3bar
          hpart += ip(kb, Q[RR_K3 * VEC + o]) / (double)t;
          J[JJ_K2 * VEC + o] = cscale(k2pb, e);                    // k2bar (partial)
          J[JJ_K1P * VEC + o] = cscale(k1ppb, e);                  // k1'bar (partial)
          J[JJ_XB * VEC + o] = cscale(x2b, e);                     // xbar (partial)
        } break;
        case AJ43_S3: {     // Y3 = x + h k2/2
          J[JJ_XB * VEC + o] = cadd(J[JJ_XB * VEC + o], Xb);
          kb = cadd(J[JJ_K2 * VEC + o], cscale(cscale(Xb, h), R(0.5)));   // k2bar final
          hpart += ip(kb, Q[RR_K2 * VEC + o]) / (double)t;
        } break;
        case AJ43_S2: {     // Y2 = x + h k1'/2; then x0bar, k1bar of this attempt
          const cplx<R> xbb = cadd(J[JJ_XB * VEC + o], Xb);
          const cplx<R> k1pb = cadd(J[JJ_K1P * VEC + o], cscale(cscale(Xb, h), R(0.5)));
          const double eb = ip(k1pb, Q[RR_K1 * VEC + o]) + ip(xbb, Q[RR_X0 * VEC + o]);
          hpart += eb * (double)dedt;
          J[JJ_X0 * VEC + o] = cscale(xbb, e);
          J[JJ_K1 * VEC + o] = cscale(k1pb, e);
          feed = false;
        } break;
        default: {          // AJ43_INIT: initial k1 = t v(x0): x0bar += Xbar
          J[JJ_X0 * VEC + o] = cadd(J[JJ_X0 * VEC + o], Xb);
          feed = false;
        } break;
      }
      kb = cscale(kb, t);
    }
    // lambda = kb; the product multipliers vanish at (0,0), which the mask removes
    lam[j] = cdiv_r(kb, cky);
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) hpart += __shfl_xor_sync(0xffffffffu, hpart, o);
  if (lane == 0) p.hacc[((size_t)b * K + ky) * 2 + ch] += hpart;
  if (!feed) return;
  // unscaled inverses Re sum mult_f lam e^{ik.x} (the row pass doubles ky > 0):
  // P1bar, P2bar from channel w, P3bar from channel j
  if (ch == 0) {
    cplx<R> z0[E], z1[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      z0[j] = cscale(lam[j], prod_mult<R>(0, kx, ky));
      z1[j] = cscale(lam[j], prod_mult<R>(1, kx, ky));
    }
    fft_dit2<R, N, true>(z0, z1, s_tw, lane);
    cplx<R>* g0 = p.G + ((size_t)(b * NG + 0) * K + ky) * N;
    cplx<R>* g1 = g0 + (size_t)K * N;
#pragma unroll
    for (int j = 0; j < E; ++j) { g0[lane + 32 * j] = z0[j]; g1[lane + 32 * j] = z1[j]; }
  } else {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      lam[j] = cscale(lam[j], prod_mult<R>(2, kx, ky));
    }
    col_inverse1<R, N>(lam, p.G, NG, b, 2, ky, lane, s_tw, R(1));
  }
}

// Rejected Lawson-RK4(3) attempt in reverse: k1_next = e (e k1) ((e, e L h/2) from the attempt's record).
template <typename R>
__global__ void k_adj_reject(cplx<R>* J, int nslot, const cplx<R>* rec, double* hacc, int n, int B) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  // one warp per (b, ky) column so that hacc[b][ky] has a single writer
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= B * g.K) return;
  const int b = colid / g.K, ky = colid - b * g.K;
  cplx<R>* Jb = J + (size_t)b * nslot * VEC;
  double part = 0.0;
  for (int ch = 0; ch < 2; ++ch)
    for (int slot = lane; slot < g.M; slot += 32) {
      const size_t o = ((size_t)ch * g.K + ky) * g.M + slot;
      const cplx<R> eg = rec[RR_E * VEC + o];   // (e, e L h/2) of the attempt
      const R e = eg.x;
      const R dedt = eg.y;
      const cplx<R> k1 = rec[RR_K1 * VEC + o], k1e = cscale(k1, e);
      const cplx<R> kppb = Jb[JJ_K1 * VEC + o];
      const cplx<R> kpb = cscale(kppb, e);
      part += (rdot2(kppb.x, kppb.y, k1e.x, k1e.y) + rdot2(kpb.x, kpb.y, k1.x, k1.y)) * (double)dedt;
      Jb[JJ_K1 * VEC + o] = cscale(kpb, e);
    }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) hacc[((size_t)b * g.K + ky) * 2] += part;
}

// Head of the adjoint: from Ybar = cotangent of sym(Phi) (box, already
// -(c/n^2) rfft2(c_out)), Phibar = sym^T(Ybar) and sxbar = <Phibar, i kx Phi>
// (symmetry.py:4-25; shift_x uses masked kx).  One block per batch element.
template <typename R>
__global__ void k_adj_head(const cplx<R>* Ybar, const cplx<R>* phi, const double* sx, int sx_shared, double sy,
                           int odd, int rot, cplx<R>* Phibar, long pb_stride, double* sxbar, int n) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  const int b = blockIdx.x;
  const double s = sx[sx_shared ? 0 : b];
  const cplx<R>* Y = Ybar + (size_t)b * VEC;
  cplx<R>* P = Phibar + (size_t)b * pb_stride;
  double part = 0.0;
  for (size_t i = threadIdx.x; i < VEC; i += blockDim.x) {
    // i indexes the SOURCE mode kappa (the mode of Phi); its image is kx_out
    const int slot = i % g.M; const int ky = (i / g.M) % g.K; const int c = (int)(i / ((size_t)g.K * g.M));
    const int kap = slot_to_kx(slot, g.kmax, g.M);
    const int kout = odd ? -kap : kap;
    const int sout = kout >= 0 ? kout : kout + g.M;
    cplx<R> y = Y[((size_t)c * g.K + ky) * g.M + sout];
    if (rot) { y.y = -y.y; if (c == 1) { y.x = -y.x; y.y = -y.y; } }   // R^T = sign_c conj
    if (odd) { y.x = -y.x; y.y = -y.y; }
    const bool m = !(kap == 0 && ky == 0);
    double sn, cs;
    sincos(m ? (double)ky * sy : 0.0, &sn, &cs);
    y = cmul(mk<R>((R)cs, (R)-sn), y);
    sincos(m ? (double)kap * s : 0.0, &sn, &cs);
    y = cmul(mk<R>((R)cs, (R)-sn), y);
    P[i] = y;
    const cplx<R> ph = phi[i];
    const R km = m ? (R)kap : R(0);
    // <y, i kap phi> = Re(conj(y) * i kap phi)
    part += (double)y.x * (double)(-km * ph.y) + (double)y.y * (double)(km * ph.x);
  }
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += red[w];
    sxbar[b] = a;
  }
}

// Ybar = -(c_ky/n^2) * box  (transpose of out = base - irfft2(.))
template <typename R>
__global__ void k_box_scale_c(cplx<R>* v, long stride, int n, int B, R sign_over_n2) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  const long total = (long)B * VEC;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / VEC); const size_t o = i - (size_t)b * VEC;
    const int ky = (o / g.M) % g.K;
    cplx<R>* q = v + (size_t)b * stride + o;
    *q = cscale(*q, (ky == 0 ? R(1) : R(2)) * sign_over_n2);
  }
}

// Z = fbar0 * n^2 / c_ky (so that from_box(Z) = to_box^T(fbar0)).
template <typename R>
__global__ void k_box_to_fields_adj(const cplx<R>* fb, long stride, cplx<R>* Z, int n, int B) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  const long total = (long)B * VEC;
  const R n2 = R(n) * R(n);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / VEC); const size_t o = i - (size_t)b * VEC;
    const int ky = (o / g.M) % g.K;
    Z[i] = cscale(fb[(size_t)b * stride + o], n2 / (ky == 0 ? R(1) : R(2)));
  }
}

// g += cT vt / (2n^2) + csx vx / (2n^2)  (phase-condition transposes, loss_functions.py:124-129)
template <typename R>
__global__ void k_adj_phase(R* gfields, const R* vt, const R* vx, const double* cT, const double* csx, int n, int B) {
  const long per = 2L * n * n;
  const long total = (long)B * per;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / per); const long o = i - (long)b * per;
    gfields[i] += (R)((cT[b] * (double)vt[o] + csx[b] * (double)vx[o]) / (double)per);
  }
}

// Deterministic reduction of the [B][K][2] accumulators: out[b] = scale * sum hacc[b].
static __global__ void k_reduce_hacc(const double* hacc, int K, double scale, double* out, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  double s = 0.0;
  for (int k = 0; k < 2 * K; ++k) s += hacc[(size_t)b * 2 * K + k];
  out[b] = s * scale;
}

// Reverse segment r of several candidates' gradient sweeps, aligned at each
// candidate's end: candidate b (nseg[b] segments) works on its segment
// g = nseg[b] - 1 - r, whose start state is ckpt[g][b]; a candidate with g < 0
// is done (skipped by every launch of the segment).
template <typename R>
__global__ void k_grad_segment(cplx<R>* F, const cplx<R>* ckpt, const int* nseg, int r, StepCtl* ctl, long vec,
                               int B) {
  const long total = (long)B * vec;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / vec);
    const int g = nseg[b] - 1 - r;
    if (i % vec == 0) ctl[b].done = g < 0 ? 1 : 0;
    if (g >= 0) F[i] = ckpt[((size_t)g * B + b) * vec + (i % vec)];
  }
}

}  // namespace ecs
