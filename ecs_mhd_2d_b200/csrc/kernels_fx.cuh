// Column passes of the other fixed-step shooting modes of mismatch_RPO
// (jax_scripts/lib/loss_functions.py:48-85), sharing the row passes and the
// adaptive stepper's slot array S [B][S_NSLOT][2][K][M]:
//   FX_RK4  classic RK4 with dissipation in the right-hand side (timestepping.py:17-44)
//   FX_RK6  Lawson sixth-order RK, e = exp(h/6 L) mask (timestepping.py:83-125)
//   FX_TD4  two-derivative RK4 (timestepping.py:127-149): each step evaluates the
//           right-hand side at f and f_temp and its Jacobian-vector product there
//           (the tangent row pass on the recorded physical fields of that point)
// One launch per stage; STAGE 0 starts a run (inverse transforms of F).  Modes
// outside the box: RK4 and TDRK4 leave them unchanged (their right-hand side
// is masked), Lawson-RK6 zeroes them (masked integrating factor), as the
// reference does.
#pragma once

#include "kernels.cuh"
#include "kernels_rk43.cuh"

namespace ecs {

enum FxScheme : int { FX_RK4 = 0, FX_RK6 = 1, FX_TD4 = 2 };
// slots: F, then K1..K7 (RK4 uses K1..K3, RK6 K1..K7); TDRK4: K1, A1, FT, K2
enum FxSlot { X_F = 0, X_K1 = 1, X_A1 = 2, X_FT = 3, X_K2T = 4 };
// TDRK4 trajectory record per step (for the tangent and adjoint): the step's
// start state, k1, a1, f_temp, k2, a2.
enum TdRec { TR_F = 0, TR_K1, TR_A1, TR_FT, TR_K2, TR_A2, TR_NREC };

template <typename R>
struct ColFxParams {
  const cplx<R>* H;     // [B][NH][K][N]
  cplx<R>* G;           // [B][NG][K][N]
  cplx<R>* S;           // [B][S_NSLOT][2][K][M]
  const R* Etab;        // [B][2][K][M] e = exp(h/6 L) mask (RK6)
  const StepCtl* ctl;   // [B] (h)
  const cplx<R>* fhat;  // [K][M]
  const cplx<R>* tw;
  R nu, eta;
  int B, produce;
  cplx<R>* rec;         // linearisation (batch 1): record of this step, or null: TDRK4 [TR_NREC][2][K][M];
                        // RK4 / Lawson-RK6 [f0, k_1..k_S, x_2..x_S] (see kernels_fxl.cuh)
};

template <int SCHEME, int STAGE> struct FxTraits {
  // the right-hand side entering this stage: 0 none, 1 full (forcing), 2 Jacobian-vector product (no forcing)
  static constexpr int rhs = STAGE == 0 ? 0 : (SCHEME == FX_TD4 && (STAGE == 2 || STAGE == 4)) ? 2 : 1;
  static constexpr int last = SCHEME == FX_RK4 ? 4 : SCHEME == FX_RK6 ? 8 : 4;
};

template <typename R, int N, int SCHEME, int STAGE>
__global__ void __launch_bounds__(128) k_col_fx(ColFxParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  using Tr = FxTraits<SCHEME, STAGE>;
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  const int c = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;   // one warp per (b, ky, channel)
  const R h = (R)p.ctl[b].h;
  const R coeff = c == 0 ? p.nu : p.eta;
  cplx<R>* S = p.S + (size_t)b * S_NSLOT * VEC;
  const R* Et = p.Etab + (size_t)b * VEC;
  cplx<R> r[E];
  if (Tr::rhs) col_load_rhs<R, N>(p.H, b, c, ky, lane, s_tw, r);
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    x[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const size_t o = ((size_t)c * K + ky) * M + slot;
    auto Q = [&](int q) -> cplx<R>& { return S[q * VEC + o]; };
    const R L = diss_L<R>(kx, ky, coeff);   // masked: zero at (0,0)
    cplx<R> v = mk<R>(0, 0);
    if (Tr::rhs) {
      v = r[j];
      if (Tr::rhs == 1 && c == 0 && !(kx == 0 && ky == 0)) v = cadd(v, p.fhat[ky * M + slot]);
    }
    cplx<R> xin = mk<R>(0, 0);
    if (STAGE == 0) {
      xin = Q(X_F);
    } else if (SCHEME == FX_RK4) {
      // v_fn includes dissipation L x at the stage input x (loss_functions.py:53, mhd_jax.py:171-173)
      const cplx<R> f = Q(X_F);
      cplx<R> xs = f;
      if (STAGE == 2) xs = cadd(f, cdiv_k<2>(Q(X_K1)));
      if (STAGE == 3) xs = cadd(f, cdiv_k<2>(Q(X_K1 + 1)));
      if (STAGE == 4) xs = cadd(f, Q(X_K1 + 2));
      const cplx<R> k = cscale(cadd(v, cscale(xs, L)), h);            // timestepping.py:40-43
      if (p.rec) {   // record: f0, k_s, x_{s+1}
        if (STAGE == 1) p.rec[o] = f;
        p.rec[STAGE * VEC + o] = k;
      }
      if (STAGE < 4) {
        Q(X_K1 + STAGE - 1) = k;
        xin = STAGE < 3 ? cadd(f, cdiv_k<2>(k)) : cadd(f, k);
        if (p.rec) p.rec[(4 + STAGE) * VEC + o] = xin;
      } else {
        const cplx<R> fn = cadd(cadd(cadd(cadd(f, cdiv_k<6>(Q(X_K1))), cdiv_k<3>(Q(X_K1 + 1))),
                                     cdiv_k<3>(Q(X_K1 + 2))), cdiv_k<6>(k));   // :44
        Q(X_F) = fn;
        xin = fn;
      }
    } else if (SCHEME == FX_RK6) {
      const R e = Et[o];
      const cplx<R> k = cscale(v, h);
      auto K_ = [&](int s) -> cplx<R>& { return Q(X_K1 + s - 1); };
      auto scale_all = [&](int upto) {   // f, k1..k_upto *= e
        Q(X_F) = cscale(Q(X_F), e);
        for (int s = 1; s <= upto; ++s) K_(s) = cscale(K_(s), e);
      };
      if (p.rec) {   // record: f0, k_s (before any factor)
        if (STAGE == 1) p.rec[o] = Q(X_F);
        p.rec[STAGE * VEC + o] = k;
      }
      switch (STAGE) {
        case 1:   // :110-112
          K_(1) = k; scale_all(1);
          xin = cadd(Q(X_F), cdiv_k<6>(K_(1)));
          break;
        case 2:   // :113
          K_(2) = k;
          xin = cadd(cadd(Q(X_F), cdiv_k<12>(K_(1))), cdiv_k<12>(K_(2)));
          break;
        case 3:   // :114-115
          K_(3) = k; scale_all(3);
          xin = cadd(csub(Q(X_F), cdiv_k<33>(cscale(K_(2), R(4)))), cdiv_k<11>(cscale(K_(3), R(5))));
          break;
        case 4:   // :116-117
          K_(4) = k; scale_all(4);
          xin = cadd(csub(csub(Q(X_F), cdiv_k<4>(K_(1))), cdiv_k<44>(cscale(K_(2), R(29)))),
                     cdiv_k<22>(cscale(K_(3), R(31))));
          break;
        case 5:   // :118-119
          K_(5) = k; scale_all(5);
          xin = cadd(cadd(csub(cadd(cadd(Q(X_F), cdiv_k<11>(cscale(K_(1), R(3)))), cdiv_k<33>(cscale(K_(2), R(8)))),
                               cdiv_k<11>(cscale(K_(3), R(4)))), cdiv_k<11>(K_(4))),
                     cdiv_k<33>(cscale(K_(5), R(14))));
          break;
        case 6:   // :120-121
          K_(6) = k; scale_all(6);
          xin = cadd(csub(cadd(cadd(csub(csub(Q(X_F), cdiv_k<48>(cscale(K_(1), R(17)))), cdiv_k<12>(cscale(K_(2), R(5)))),
                                    K_(3)), K_(4)), cdiv_k<12>(cscale(K_(5), R(13)))),
                     cdiv_k<16>(cscale(K_(6), R(11))));
          break;
        case 7:   // :122-123
          K_(7) = k; scale_all(7);
          xin = cadd(csub(cadd(csub(csub(cadd(cadd(Q(X_F), cdiv_k<39>(cscale(K_(1), R(20)))),
                                                  cdiv_k<39>(cscale(K_(2), R(12)))),
                                             cdiv_k<39>(cscale(K_(3), R(31)))), cdiv_k<39>(K_(4))),
                                   cdiv_k<39>(cscale(K_(5), R(34)))), cdiv_k<39>(cscale(K_(6), R(11)))),
                     cdiv_k<39>(cscale(K_(7), R(16))));
          break;
        default: {   // 8: :124
          const R c1 = R(13) / R(200), c3 = R(4) / R(25), c4 = R(11) / R(40);
          const cplx<R> fn = cadd(cadd(cadd(Q(X_F), cscale(cadd(K_(1), k), c1)), cscale(cadd(K_(3), K_(7)), c3)),
                                  cscale(cadd(K_(4), K_(6)), c4));
          Q(X_F) = fn;
          xin = fn;
        } break;
      }
      if (p.rec && STAGE < 8) p.rec[(8 + STAGE) * VEC + o] = xin;   // the stage input x_{s+1}
    } else {   // FX_TD4, timestepping.py:137-144; v_fn and its derivative include dissipation
      switch (STAGE) {
        case 1: {   // k1 = h v(f); next: the transforms of k1 (tangent input of jac(f, k1))
          const cplx<R> k1 = cscale(cadd(v, cscale(Q(X_F), L)), h);
          Q(X_K1) = k1;
          if (p.rec) { p.rec[TR_F * VEC + o] = Q(X_F); p.rec[TR_K1 * VEC + o] = k1; }
          xin = k1;
        } break;
        case 2: {   // a1 = h jac(f, k1); f_temp = f + k1/2 + a1/8
          const cplx<R> k1 = Q(X_K1);
          const cplx<R> a1 = cscale(cadd(v, cscale(k1, L)), h);
          Q(X_A1) = a1;
          const cplx<R> ft = cadd(cadd(Q(X_F), cdiv_k<2>(k1)), cdiv_k<8>(a1));
          Q(X_FT) = ft;
          if (p.rec) { p.rec[TR_A1 * VEC + o] = a1; p.rec[TR_FT * VEC + o] = ft; }
          xin = ft;
        } break;
        case 3: {   // k2 = h v(f_temp)
          const cplx<R> k2 = cscale(cadd(v, cscale(Q(X_FT), L)), h);
          Q(X_K2T) = k2;
          if (p.rec) p.rec[TR_K2 * VEC + o] = k2;
          xin = k2;
        } break;
        default: {  // a2 = h jac(f_temp, k2); f = f + k1 + a1/6 + a2/3
          const cplx<R> a2 = cscale(cadd(v, cscale(Q(X_K2T), L)), h);
          if (p.rec) p.rec[TR_A2 * VEC + o] = a2;
          const cplx<R> fn = cadd(cadd(cadd(Q(X_F), Q(X_K1)), cdiv_k<6>(Q(X_A1))), cdiv_k<3>(a2));
          Q(X_F) = fn;
          xin = fn;
        } break;
      }
    }
    x[j] = xin;
  }
  if (!p.produce) return;
  col_inverse_uv<R, N>(x, p.G, b, c, ky, lane, s_tw);
}

// ---------------------------------------------------------------------------
// TDRK4 tangent.  With the quadratic right-hand side, N'(f) x = N'(x) f, so the
// tangent of a1 = h J(f) k1 is (dh/h) a1 + h [N'(f) dk1 + N'(k1) df + L dk1]:
// one "dual" tangent row pass of two tangent field sets against two primal
// field sets.  Per step, along (df, dT):
//   dk1 = (dh/h) k1 + h J(f) df
//   da1 = (dh/h) a1 + h [N'(f) dk1 + N'(k1) df + L dk1]
//   dft = df + dk1/2 + da1/8
//   dk2 = (dh/h) k2 + h J(f_temp) dft
//   da2 = (dh/h) a2 + h [N'(f_temp) dk2 + N'(k2) dft + L dk2]
//   df' = df + dk1 + da1/6 + da2/3
// Ga holds the transforms of df / dft, Gb those of dk1 / dk2.
// ---------------------------------------------------------------------------
template <typename R>
struct RowTan2Params {
  const cplx<R>* Ga;    // [B][NG][K][N] tangent paired with phys_b
  const cplx<R>* Gb;    // [B][NG][K][N] tangent paired with phys_a
  cplx<R>* H;           // [B][NH][K][N]
  const R* phys_a;      // primal point (f or f_temp), B_x/B_y with the mean field: [N][NPH][N]
  const R* phys_b;      // stage derivative (k1 or k2), no mean field: [N][NPH][N]
  const cplx<R>* tw;
  int B;
};

// Linearised products dP of one tangent (du, dv, dbx, dby) about one field set (u, v, bx, by), accumulated.
template <typename R>
__device__ __forceinline__ void acc_tan_products(R u, R v, R bx, R by, R du, R dv, R dbx, R dby, cplx<R>& W, R& p3) {
  W.x += R(2) * ((u * du - v * dv) - (bx * dbx - by * dby));   // dP1
  W.y += (bx * dby + by * dbx) - (u * dv + v * du);            // dP2
  p3 += (u * dby + by * du) - (v * dbx + bx * dv);             // dP3
}

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_tan2(RowTan2Params<R> p) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_Ga = s_tw + fft_smem(N, XT);
  cplx<R>* s_Gb = s_Ga + NG * K * (XT + 1);
  cplx<R>* s_H = s_Gb + NG * K * (XT + 1);
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = x0 + w;
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  load_tile<R, N, XT>(s_Ga, p.Ga + (size_t)b * NG * K * N, NG * K, x0);
  load_tile<R, N, XT>(s_Gb, p.Gb + (size_t)b * NG * K * N, NG * K, x0);
  __syncthreads();
  cplx<R> W[E];
  R p3[E];
#pragma unroll
  for (int j = 0; j < E; ++j) { W[j] = mk<R>(0, 0); p3[j] = R(0); }
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {   // pass 0: Gb about phys_a; pass 1: Ga about phys_b
    const cplx<R>* sg = pass == 0 ? s_Gb : s_Ga;
    const R* ph = phys_row<R, N>(pass == 0 ? p.phys_a : p.phys_b, x);
    cplx<R> duv[E], dbb[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int q = lane + 32 * j;
      duv[j] = packed_pair<R, N, XT>(sg + 0 * K * (XT + 1), sg + 1 * K * (XT + 1), q, w);
      dbb[j] = packed_pair<R, N, XT>(sg + 2 * K * (XT + 1), sg + 3 * K * (XT + 1), q, w);
    }
    fft_dif2<R, N, true>(duv, dbb, s_tw, lane);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = lane + 32 * j;
      acc_tan_products<R>(ph[e], ph[N + e], ph[2 * N + e], ph[3 * N + e], duv[j].x, duv[j].y, dbb[j].x, dbb[j].y,
                          W[j], p3[j]);
    }
  }
  cplx<R> Z[E];
#pragma unroll
  for (int j = 0; j < E; ++j) Z[j] = mk<R>(p3[j], R(0));
  fft_dit2<R, N, false>(W, Z, s_tw, lane);
  split_store<R, N, XT>(W, s_H, s_H + K * (XT + 1), w, lane);
  store_one<R, N, XT>(Z, s_H + 2 * K * (XT + 1), w, lane);
  __syncthreads();
  store_tile<R, N, XT>(p.H + (size_t)b * NH * K * N, s_H, NH * K, x0);
}

enum TdTanSlot { DT_F = 0, DT_K1, DT_A1, DT_FT, DT_K2, DT_NSLOT };

template <typename R>
struct ColTdjParams {
  const cplx<R>* H;     // [B][NH][K][N]
  cplx<R>* Ga;          // [B][NG][K][N]
  cplx<R>* Gb;          // [B][NG][K][N]
  cplx<R>* D;           // tangent slots [B][nslot][2][K][M]
  int nslot;
  const cplx<R>* rec;   // primal record of this step [TR_NREC][2][K][M]
  const double* dT;     // [B]
  double h, dscale;     // dh = dT * dscale
  const cplx<R>* tw;
  R nu, eta;
  int B, produce;
};

template <typename R, int N, int STAGE>
__global__ void __launch_bounds__(128) k_col_tdj(ColTdjParams<R> p) {
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
  const int c = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;
  cplx<R>* D = p.D + (size_t)b * p.nslot * VEC;
  const cplx<R>* Q = p.rec;
  const R h = (R)p.h;
  const R dpar = (R)(p.dT[b] * p.dscale);   // dh
  const R coeff = c == 0 ? p.nu : p.eta;
  cplx<R> r[E];
  if (STAGE != 0) col_load_rhs<R, N>(p.H, b, c, ky, lane, s_tw, r);
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    x[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const size_t o = ((size_t)c * K + ky) * M + slot;
    const R L = diss_L<R>(kx, ky, coeff);
    auto Dq = [&](int q) -> cplx<R>& { return D[q * VEC + o]; };
    // d(h X) = (dh/h) (h X) + h dX, with the recorded h X and dX = r + L dx (no forcing)
    auto dk = [&](int q, cplx<R> dxin) { return cadd(cscale(Q[q * VEC + o], dpar / h), cscale(cadd(r[j], cscale(dxin, L)), h)); };
    cplx<R> xin = mk<R>(0, 0);
    switch (STAGE) {
      case 0: xin = Dq(DT_F); break;
      case 1: { const cplx<R> dk1 = dk(TR_K1, Dq(DT_F)); Dq(DT_K1) = dk1; xin = dk1; } break;
      case 2: {
        const cplx<R> dk1 = Dq(DT_K1);
        const cplx<R> da1 = dk(TR_A1, dk1);
        Dq(DT_A1) = da1;
        const cplx<R> dft = cadd(cadd(Dq(DT_F), cdiv_k<2>(dk1)), cdiv_k<8>(da1));
        Dq(DT_FT) = dft;
        xin = dft;
      } break;
      case 3: { const cplx<R> dk2 = dk(TR_K2, Dq(DT_FT)); Dq(DT_K2) = dk2; xin = dk2; } break;
      default: {
        const cplx<R> da2 = dk(TR_A2, Dq(DT_K2));
        const cplx<R> dfn = cadd(cadd(cadd(Dq(DT_F), Dq(DT_K1)), cdiv_k<6>(Dq(DT_A1))), cdiv_k<3>(da2));
        Dq(DT_F) = dfn;
        xin = dfn;
      } break;
    }
    x[j] = xin;
  }
  if (!p.produce) return;
  // dk1, dk2 go to Gb (paired with the point f / f_temp); df, dft, df' to Ga
  col_inverse_uv<R, N>(x, (STAGE == 1 || STAGE == 3) ? p.Gb : p.Ga, b, c, ky, lane, s_tw);
}

// ---------------------------------------------------------------------------
// TDRK4 adjoint.  Reverse of one step (lambda = h xbar is the input of each
// adjoint row pass; N'(x)^T from the transposed product chain of kernels_adj.cuh):
//   seed: a2bar = fbar'/3, k1bar = fbar', a1bar = fbar'/6, fbar = fbar'
//   dual pass, lambda = h a2bar at (f_temp, k2):  k2bar = N'(ft)^T lambda + h L a2bar,  ftbar = N'(k2)^T lambda
//   pass, lambda = h k2bar at f_temp:             ftbar += N'(ft)^T lambda + h L k2bar
//   fbar += ftbar, k1bar += ftbar/2, a1bar += ftbar/8
//   dual pass, lambda = h a1bar at (f, k1):       k1bar += N'(f)^T lambda + h L a1bar,  fbar += N'(k1)^T lambda
//   pass, lambda = h k1bar at f:                  fbar += N'(f)^T lambda + h L k1bar
// and hbar += <a2bar, a2>/h + <k2bar, k2>/h + <a1bar, a1>/h + <k1bar, k1>/h.
// ---------------------------------------------------------------------------
template <typename R>
struct RowAdj2Params {
  const cplx<R>* G;     // [B][NG][K][N]: fields 0..2 the product cotangents of lambda (/c_ky)
  cplx<R>* Ha;          // [B][NHA][K][N]: rfft2 rows of N'(phys_a)^T
  cplx<R>* Hb;          // [B][NHA][K][N]: rfft2 rows of N'(phys_b)^T
  const R* phys_a;      // [N][NPH][N]
  const R* phys_b;      // [N][NPH][N]
  const cplx<R>* tw;
  int B;
};

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_adj2(RowAdj2Params<R> p) {
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
  load_tile<R, N, XT>(s_G, p.G + (size_t)b * NG * K * N, 3 * K, x0);
  __syncthreads();
  cplx<R> P12[E], P3[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    P12[j] = packed_pair<R, N, XT>(s_G, s_G + K * (XT + 1), lane + 32 * j, w);
    P3[j] = packed_one<R, N, XT>(s_G + 2 * K * (XT + 1), lane + 32 * j, w);
  }
  fft_dif2<R, N, true>(P12, P3, s_tw, lane);
#pragma unroll 1
  for (int pass = 0; pass < 2; ++pass) {
    const R* ph = phys_row<R, N>(pass == 0 ? p.phys_a : p.phys_b, x);
    cplx<R> A[E], Bv[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = lane + 32 * j;
      const R p1 = P12[j].x, p2 = P12[j].y, p3 = P3[j].x;
      const R u = ph[e], v = ph[N + e], bx = ph[2 * N + e], by = ph[3 * N + e];
      A[j] = mk<R>(R(2) * u * p1 - v * p2 + by * p3, -R(2) * v * p1 - u * p2 - bx * p3);     // (ubar, vbar)
      Bv[j] = mk<R>(-R(2) * bx * p1 + by * p2 - v * p3, R(2) * by * p1 + bx * p2 + u * p3);  // (Bxbar, Bybar)
    }
    fft_dit2<R, N, false>(A, Bv, s_tw, lane);
    split_store<R, N, XT>(A, s_H, s_H + K * (XT + 1), w, lane);
    split_store<R, N, XT>(Bv, s_H + 2 * K * (XT + 1), s_H + 3 * K * (XT + 1), w, lane);
    __syncthreads();
    store_tile<R, N, XT>((pass == 0 ? p.Ha : p.Hb) + (size_t)b * NHA * K * N, s_H, NHA * K, x0);
    __syncthreads();
  }
}

enum TdAdjSlot { JT_F = 0, JT_K1, JT_A1, JT_FT, JT_K2, JT_A2, JT_NSLOT };
enum TdAdjStage { TA_SEED = 0, TA_B = 1, TA_C = 2, TA_D = 3, TA_E = 4 };

template <typename R>
struct ColTdaParams {
  const cplx<R>* Ha;    // [B][NHA][K][N]
  const cplx<R>* Hb;    // [B][NHA][K][N] (dual passes)
  cplx<R>* G;           // [B][NG][K][N] (fields 0..2 written)
  cplx<R>* J;           // adjoint slots [B][nslot][2][K][M]
  int nslot;
  const cplx<R>* rec;   // primal record of this step [TR_NREC][2][K][M]
  double* hacc;         // [B][K][2]
  double h;
  const cplx<R>* tw;
  R nu, eta;
  int B;
};

// (c_ky/n^2) sum_m (-i mu_m) rfft2 of the adjoint rows of channel c in H: the box cotangent N'(P)^T lambda.
template <typename R, int N>
__device__ __forceinline__ void col_adj_xb(const cplx<R>* __restrict__ H, int b, int c, int ky, int lane,
                                           const cplx<R>* s_tw, cplx<R> (&xb)[N / 32]) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  const cplx<R>* h0 = H + ((size_t)(b * NHA + 2 * c) * K + ky) * N;
  const cplx<R>* h1 = h0 + (size_t)K * N;
  cplx<R> v1[E];
#pragma unroll
  for (int j = 0; j < E; ++j) { xb[j] = h0[lane + 32 * j]; v1[j] = h1[lane + 32 * j]; }
  fft_dif2<R, N, false>(xb, v1, s_tw, lane);
  const R cky = ky == 0 ? R(1) : R(2);
  const R inv_n2 = R(1) / (R(N) * R(N));
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int kx = pos_to_k(spec_pos<N>(lane, j), N);
    xb[j] = cscale(cadd(cimul(xb[j], -spectral_mu<R>(2, kx, ky)), cimul(v1[j], -spectral_mu<R>(3, kx, ky))), cky * inv_n2);
  }
}

// Inverse column transforms of lambda/c_ky times the product multipliers: the
// product cotangents P1bar, P2bar (channel w) or P3bar (channel j) in G.
template <typename R, int N>
__device__ __forceinline__ void col_adj_emit(cplx<R> (&lam)[N / 32], cplx<R>* __restrict__ G, int b, int c, int ky,
                                             int lane, const cplx<R>* s_tw) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  if (c == 0) {
    cplx<R> z0[E], z1[E];
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      z0[j] = cscale(lam[j], prod_mult<R>(0, kx, ky));
      z1[j] = cscale(lam[j], prod_mult<R>(1, kx, ky));
    }
    fft_dit2<R, N, true>(z0, z1, s_tw, lane);
    cplx<R>* g0 = G + ((size_t)(b * NG + 0) * K + ky) * N;
    cplx<R>* g1 = g0 + (size_t)K * N;
#pragma unroll
    for (int j = 0; j < E; ++j) { g0[lane + 32 * j] = z0[j]; g1[lane + 32 * j] = z1[j]; }
  } else {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      lam[j] = cscale(lam[j], prod_mult<R>(2, kx, ky));
    }
    col_inverse1<R, N>(lam, G, NG, b, 2, ky, lane, s_tw, R(1));
  }
}

template <typename R, int N, int STAGE>
__global__ void __launch_bounds__(128) k_col_tda(ColTdaParams<R> p) {
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
  const int c = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;
  cplx<R>* J = p.J + (size_t)b * p.nslot * VEC;
  const cplx<R>* Q = p.rec;
  const R h = (R)p.h;
  const R coeff = c == 0 ? p.nu : p.eta;
  const R cky = ky == 0 ? R(1) : R(2);
  cplx<R> xa[E], xbb[E];
  if (STAGE != TA_SEED) col_adj_xb<R, N>(p.Ha, b, c, ky, lane, s_tw, xa);
  if (STAGE == TA_B || STAGE == TA_D) col_adj_xb<R, N>(p.Hb, b, c, ky, lane, s_tw, xbb);
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
    auto Jq = [&](int q) -> cplx<R>& { return J[q * VEC + o]; };
    auto ip = [&](cplx<R> a, cplx<R> bb) { return (double)a.x * (double)bb.x + (double)a.y * (double)bb.y; };
    cplx<R> kb = mk<R>(0, 0);   // cotangent whose h-multiple feeds the next adjoint pass
    switch (STAGE) {
      case TA_SEED: {
        const cplx<R> fb = Jq(JT_F);
        const cplx<R> a2b = cdiv_k<3>(fb);
        Jq(JT_A2) = a2b; Jq(JT_K1) = fb; Jq(JT_A1) = cdiv_k<6>(fb);
        hpart += ip(a2b, Q[TR_A2 * VEC + o]) / (double)h;
        kb = a2b;
      } break;
      case TA_B: {
        const cplx<R> k2b = cadd(xa[j], cscale(Jq(JT_A2), h * L));
        Jq(JT_K2) = k2b; Jq(JT_FT) = xbb[j];
        hpart += ip(k2b, Q[TR_K2 * VEC + o]) / (double)h;
        kb = k2b;
      } break;
      case TA_C: {
        const cplx<R> ftb = cadd(cadd(Jq(JT_FT), xa[j]), cscale(Jq(JT_K2), h * L));
        Jq(JT_F) = cadd(Jq(JT_F), ftb);
        Jq(JT_K1) = cadd(Jq(JT_K1), cdiv_k<2>(ftb));
        const cplx<R> a1b = cadd(Jq(JT_A1), cdiv_k<8>(ftb));
        Jq(JT_A1) = a1b;
        hpart += ip(a1b, Q[TR_A1 * VEC + o]) / (double)h;
        kb = a1b;
      } break;
      case TA_D: {
        const cplx<R> k1b = cadd(cadd(Jq(JT_K1), xa[j]), cscale(Jq(JT_A1), h * L));
        Jq(JT_K1) = k1b;
        Jq(JT_F) = cadd(Jq(JT_F), xbb[j]);
        hpart += ip(k1b, Q[TR_K1 * VEC + o]) / (double)h;
        kb = k1b;
      } break;
      default: {   // TA_E: the cotangent of the step's start state
        Jq(JT_F) = cadd(cadd(Jq(JT_F), xa[j]), cscale(Jq(JT_K1), h * L));
      } break;
    }
    lam[j] = cdiv_r(cscale(kb, h), cky);
  }
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) hpart += __shfl_xor_sync(0xffffffffu, hpart, off);
  if (lane == 0) p.hacc[((size_t)b * K + ky) * 2 + c] += hpart;
  if (STAGE == TA_E) return;
  col_adj_emit<R, N>(lam, p.G, b, c, ky, lane, s_tw);
}

// Box entries back into the full half spectrum, leaving every other entry as it is
// (RK4 / TDRK4 carry the modes outside the box unchanged).
template <typename R>
__global__ void k_scatter_box_keep(const cplx<R>* box, cplx<R>* full, int n, int B) {
  const Geom g = make_geom(n);
  const int nh = n / 2 + 1;
  const long total = (long)B * 2 * n * nh;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ky = i % nh; const long r = i / nh; const int pos = r % n; const long bc = r / n;
    const int slot = (ky < g.K) ? pos_to_slot(pos, n, g.kmax, g.M) : -1;
    if (slot >= 0) full[i] = box[(bc * g.K + ky) * g.M + slot];
  }
}

// Recurrence matrix of snapshots (jax_scripts/generate_turbulence.py:136-146):
// dist[j][i] = || |fs_j| - |fs_i| ||_2 over the len complex entries of a
// snapshot (spectral magnitudes: blind to translations).  One block per pair
// j >= i (the matrix is symmetric), FP64 accumulation, a fixed-order tree.
template <typename R>
__global__ void k_recurrence(const cplx<R>* fs, int S, long len, double* dist) {
  const int i = blockIdx.x, j = blockIdx.y;
  if (j < i) return;
  const cplx<R>* a = fs + (size_t)j * len;
  const cplx<R>* b = fs + (size_t)i * len;
  double acc = 0.0;
  for (long k = threadIdx.x; k < len; k += blockDim.x) {
    const double d = hypot((double)a[k].x, (double)a[k].y) - hypot((double)b[k].x, (double)b[k].y);
    acc += d * d;
  }
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    const double r = sqrt(t);
    dist[(size_t)j * S + i] = r;
    dist[(size_t)i * S + j] = r;
  }
}

// e = exp(h/div L) mask and h = (T/nc)/ms per batch element (timestepping.py:69-72, :105-108).
template <typename R>
__global__ void k_fx_setup(const double* T, int nc, int ms, int div, StepCtl* ctl, R* Etab, int n, double nu,
                           double eta, int B) {
  const Geom g = make_geom(n);
  const long per = 2L * g.K * g.M;
  const long total = (long)B * per;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / per);
    const double tseg = T[b] / (double)nc;
    const R h = (R)(tseg / (double)ms);
    if (i % per == 0) { ctl[b].t = tseg; ctl[b].h = (double)h; }
    const int slot = i % g.M; const long r = i / g.M; const int ky = r % g.K; const int c = (r / g.K) & 1;
    const int kx = slot_to_kx(slot, g.kmax, g.M);
    const R L = diss_L<R>(kx, ky, (R)(c == 0 ? nu : eta));
    const bool msk = !(kx == 0 && ky == 0);
    Etab[i] = msk ? exp(h / R(div) * L) : R(0);
  }
}

}  // namespace ecs
