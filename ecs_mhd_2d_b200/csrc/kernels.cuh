// Hot-path kernels of the pseudo-spectral MHD right-hand side and the Lawson
// steppers.  One right-hand-side evaluation (reference: state_vel,
// jax_scripts/lib/mhd_jax.py:105-175) is split into two passes around the two
// transposes of a 2D FFT.
//
// Nonlinear terms.  The reference forms
//   dw/dt = -(u.grad w) + (B.grad j) + f,   dj/dt = k^2 rfft2(u B_y - v B_x)
// from 8 physical fields (the x and y derivatives of w and j and the uncurled
// velocities u, v, B_x, B_y, B with the mean field b0).  For divergence-free u
// and B with w = dv/dx - du/dy (and j likewise from B) the advection terms
// equal Basdevant's form
//   u.grad w = d_xy(v^2 - u^2) + (d_xx - d_yy)(u v)
// so that, with
//   P1 = (u^2 - v^2) - (B_x^2 - B_y^2),  P2 = B_x B_y - u v,  P3 = u B_y - v B_x,
//   dw/dt = mask (-kx ky P1^ + (ky^2 - kx^2) P2^ + f^),   dj/dt = k^2 mask P3^.
// Products of two fields on the 2/3-dealiased box alias only onto modes outside
// the box, so the retained modes of both forms are equal in exact arithmetic;
// this form needs 4 physical fields instead of 8 and 7 column transforms
// instead of 10.
//
//   column pass (one warp per (batch, ky, channel), x contiguous):
//     [forward FFTs along x of the product rows of the previous RHS: P1, P2
//      (channel w) or P3 (channel j)]
//     -> spectral epilogue (multipliers, dealias mask, forcing, stepper stage algebra)
//     -> stage input -> the two uncurling multipliers i ky/k^2, -i kx/k^2
//        -> 2 inverse FFTs along x -> G (u, v or B_x, B_y)
//   row pass (one warp per physical row x, CTA = XT rows staged in shared memory):
//     4 half-spectra rows of G -> 2 complex inverse FFTs (two real fields
//     packed per transform) -> P1, P2, P3 -> 2 forward FFTs -> split -> H
//
// The box layout and intermediate layouts are documented in common.cuh.
#pragma once

#include "common.cuh"
#include "fft.cuh"

#include <cooperative_groups.h>

namespace ecs {

// Field counts of the intermediate arrays (per batch element).
constexpr int NG = 4;    // G[b][NG][K][N]: inverse column transforms of u, v, B_x, B_y (no mean field)
constexpr int NH = 3;    // H[b][NH][K][N]: row transforms of P1, P2, P3
constexpr int NPH = 4;   // physical record rows: u, v, B_x + b0x, B_y + b0y
constexpr int NHA = 4;   // adjoint H[b][NHA][K][N]: row transforms of the cotangents of u, v, B_x, B_y

// ---------------------------------------------------------------------------
// spectral helpers
// ---------------------------------------------------------------------------

// Multiplier mu for field m in {0:x, 1:y, 2:u, 3:v} at integer (kx, ky) inside
// the box, matching mhd_jax.py:83-90 (to_u = ky/k^2, to_v = -kx/k^2, masked).
template <typename R>
__device__ __forceinline__ R spectral_mu(int m, int kx, int ky) {
  if (kx == 0 && ky == 0) return R(0);
  const R rkx = (R)kx, rky = (R)ky;
  const R ksq = rkx * rkx + rky * rky;
  switch (m) {
    case 0: return rkx;
    case 1: return rky;
    case 2: return rky / ksq;
    default: return (-rkx) / ksq;
  }
}

// (kx^2 + ky^2) * mask with masked kx, ky (mhd_jax.py:154).
template <typename R>
__device__ __forceinline__ R ksq_masked(int kx, int ky) {
  if (kx == 0 && ky == 0) return R(0);
  const R rkx = (R)kx, rky = (R)ky;
  return rkx * rkx + rky * rky;
}

// Dissipation L = -(kx^2+ky^2) * coeff (mhd_jax.py:97-102), zero at (0,0).
template <typename R>
__device__ __forceinline__ R diss_L(int kx, int ky, R coeff) {
  return (-ksq_masked<R>(kx, ky)) * coeff;
}

// Multiplier of the transformed product row f in {0: P1, 1: P2, 2: P3} in the
// nonlinear time derivative: -kx ky, ky^2 - kx^2 (channel w), k^2 (channel j).
// Integer arithmetic, exact; zero at (0,0), which the mask removes.
template <typename R>
__device__ __forceinline__ R prod_mult(int f, int kx, int ky) {
  const int m = f == 0 ? -kx * ky : f == 1 ? ky * ky - kx * kx : kx * kx + ky * ky;
  return (R)m;
}

// ---------------------------------------------------------------------------
// column-pass building blocks (one warp per (batch, ky, channel))
// ---------------------------------------------------------------------------

// Nonlinear time derivative of channel ch (without forcing) at every position
// of the column ky, bit-reversed slot order, from the product rows in H:
//   ch 0: -kx ky rfft2(P1) + (ky^2 - kx^2) rfft2(P2)  (two transforms in lockstep),
//   ch 1: k^2 rfft2(P3).
// The same from the product rows given directly: h0, h1 = the P1, P2 rows of
// column ky (ch 0), or h0 = its P3 row (ch 1); global or shared memory.
template <typename R, int N>
__device__ __forceinline__ void col_rhs_rows(const cplx<R>* h0, const cplx<R>* h1, int ch, int ky, int lane,
                                             const cplx<R>* s_tw, cplx<R> (&v)[N / 32]) {
  constexpr int E = N / 32;
  if (ch == 0) {
    cplx<R> r[E];
#pragma unroll
    for (int j = 0; j < E; ++j) { v[j] = h0[lane + 32 * j]; r[j] = h1[lane + 32 * j]; }
    fft_dif2<R, N, false>(v, r, s_tw, lane);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      const R m0 = prod_mult<R>(0, kx, ky), m1 = prod_mult<R>(1, kx, ky);
      v[j] = mk<R>(fpp(m0, v[j].x, m1, r[j].x), fpp(m0, v[j].y, m1, r[j].y));
    }
  } else {
#pragma unroll
    for (int j = 0; j < E; ++j) v[j] = h0[lane + 32 * j];
    fft_dif<R, N, false>(v, s_tw, lane);
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int kx = pos_to_k(spec_pos<N>(lane, j), N);
      v[j] = cscale(v[j], prod_mult<R>(2, kx, ky));
    }
  }
}

template <typename R, int N>
__device__ __forceinline__ void col_load_rhs(const cplx<R>* __restrict__ H, int b, int ch, int ky, int lane,
                                             const cplx<R>* s_tw, cplx<R> (&v)[N / 32]) {
  constexpr int K = (N - 1) / 3 + 1;
  const cplx<R>* h0 = H + ((size_t)(b * NH + (ch == 0 ? 0 : 2)) * K + ky) * N;
  col_rhs_rows<R, N>(h0, h0 + (size_t)K * N, ch, ky, lane, s_tw, v);
}

// Stage input x of channel c (bit-reversed slot order) -> its two uncurled
// fields i (ky/k^2) x and i (-kx/k^2) x (mhd_jax.py:140-141) transformed along
// x in lockstep, scaled by 1/n^2, to G fields 2c and 2c+1.
template <typename R, int N>
__device__ __forceinline__ void col_uv_transform(const cplx<R> (&x)[N / 32], int ky, int lane, const cplx<R>* s_tw,
                                                 cplx<R> (&wu)[N / 32], cplx<R> (&wv)[N / 32]) {
  constexpr int E = N / 32;
  const R inv_n2 = R(1) / (R(N) * R(N));
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int kx = pos_to_k(spec_pos<N>(lane, j), N);
    wu[j] = cscale(cimul(x[j], spectral_mu<R>(2, kx, ky)), inv_n2);
    wv[j] = cscale(cimul(x[j], spectral_mu<R>(3, kx, ky)), inv_n2);
  }
  fft_dit2<R, N, true>(wu, wv, s_tw, lane);
}

// Cluster-resident passes (kernels_chain.cuh): a cluster of N / XT CTAs holds
// one state; CTA r keeps the G tile of physical rows x in [XT r, XT r + XT)
// (NG K rows of pitch XT + 1, at the same shared-memory offset in every CTA).

// The two G rows of col_inverse_uv written into the cluster's G tiles instead of
// global memory: position x goes to CTA x / XT, tile rows (2c) K + ky (u) and
// (2c + 1) K + ky (v), column x % XT.  `tile` is this CTA's tile.
template <typename R, int N, int XT>
__device__ __forceinline__ void col_uv_to_tiles(const cplx<R> (&wu)[N / 32], const cplx<R> (&wv)[N / 32],
                                                cplx<R>* tile, int c, int ky, int lane) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int x = lane + 32 * j;
    cplx<R>* t = cl.map_shared_rank(tile, (unsigned)(x / XT));
    t[((2 * c) * K + ky) * (XT + 1) + x % XT] = wu[j];
    t[((2 * c + 1) * K + ky) * (XT + 1) + x % XT] = wv[j];
  }
}

// The NH K rows of a row pass's H tile (pitch XT + 1, physical rows x0 ..
// x0 + XT - 1) sent to the warps of the cluster that transform them: row
// (f, ky) feeds column c = 2 ky + (f == 2) of the column passes, which warp
// c / CL of CTA c % CL holds (CL = N / XT CTAs) in its two rows of N at
// hcols + (c / CL) 2 N: P1, P2 (channel 0), or P3 in the first (channel 1).
template <typename R, int N, int XT>
__device__ __forceinline__ void scatter_h_tile(const cplx<R>* s_H, cplx<R>* hcols, int x0) {
  constexpr int K = (N - 1) / 3 + 1;
  constexpr int CL = N / XT;
  cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
  for (int i = threadIdx.x; i < NH * K * XT; i += blockDim.x) {
    const int rr = i / XT, xt = i - rr * XT;
    const int f = rr / K, ky = rr - f * K;
    const int c = 2 * ky + (f == 2 ? 1 : 0);
    cplx<R>* dst = cl.map_shared_rank(hcols, (unsigned)(c % CL));
    dst[((c / CL) * 2 + (f == 2 ? 0 : f)) * N + x0 + xt] = s_H[rr * (XT + 1) + xt];
  }
}

template <typename R, int N>
__device__ __forceinline__ void col_inverse_uv(const cplx<R> (&x)[N / 32], cplx<R>* __restrict__ G, int b, int c,
                                               int ky, int lane, const cplx<R>* s_tw) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  cplx<R> wu[E], wv[E];
  col_uv_transform<R, N>(x, ky, lane, s_tw, wu, wv);
  cplx<R>* gu = G + ((size_t)(b * NG + 2 * c) * K + ky) * N;
  cplx<R>* gv = gu + (size_t)K * N;
#pragma unroll
  for (int j = 0; j < E; ++j) { gu[lane + 32 * j] = wu[j]; gv[lane + 32 * j] = wv[j]; }
}

// One plain inverse transform along x of a box column, scaled, to field f of
// G[b] (nf fields per batch element).
template <typename R, int N>
__device__ __forceinline__ void col_inverse1(const cplx<R> (&x)[N / 32], cplx<R>* __restrict__ G, int nf, int b,
                                             int f, int ky, int lane, const cplx<R>* s_tw, R scale) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  cplx<R> w[E];
#pragma unroll
  for (int j = 0; j < E; ++j) w[j] = cscale(x[j], scale);
  fft_dit<R, N, true>(w, s_tw, lane);
  cplx<R>* gout = G + ((size_t)(b * nf + f) * K + ky) * N;
#pragma unroll
  for (int j = 0; j < E; ++j) gout[lane + 32 * j] = w[j];
}

// ---------------------------------------------------------------------------
// Column pass of the forward RHS fused with the Lawson-RK4 stage algebra
// (reference: timestepping.lawson_rk4, jax_scripts/lib/timestepping.py:69-80).
// ---------------------------------------------------------------------------

// Lawson-RK4 record per step (box vectors): stage input X1 = F, stage
// derivatives k1..k4 (before twiddles) and stage inputs X2..X4.
enum Rk4Rec { Q_F = 0, Q_K1, Q_K2, Q_K3, Q_K4, Q_X2, Q_X3, Q_X4, Q_NREC };

enum ColStage : int {
  COL_START = 0,     // no RHS input; stage input = F (start of a step)
  COL_RK4_S1 = 1,    // finish k1, stage input X2
  COL_RK4_S2 = 2,    // finish k2, stage input X3
  COL_RK4_S3 = 3,    // finish k3, stage input X4
  COL_RK4_S4 = 4,    // finish k4 (state update), stage input X1 of next step
  COL_PLAIN = 5,     // finish RHS: OUT = v (+ L f0 if diss)   [state_vel]
};

template <typename R>
struct ColParams {
  const cplx<R>* H;      // [B][NH][K][N]
  cplx<R>* G;            // [B][NG][K][N]
  cplx<R>* F;            // [B][2][K][M]   state / accumulator
  cplx<R>* A1;           // [B][2][K][M]   e*k1
  cplx<R>* K2;           // [B][2][K][M]   k2
  cplx<R>* OUT;          // [B][2][K][M]   COL_PLAIN output
  const R* Etab;         // [B][2][K][M]   exp(h/2 L) * mask
  const StepCtl* ctl;    // [B]
  const cplx<R>* fhat;   // [K][M] box spectrum of the forcing (omega only)
  const cplx<R>* tw;     // [N/2]
  R nu, eta;
  int B;
  int stage;
  int produce;           // write G for the stage input
  int diss;              // COL_PLAIN: add L f (f = F)
  cplx<R>* rec;          // optional record of this step: [Q_NREC][2][K][M] per batch element
  long rec_bstride;      // elements between batch elements in rec
  int use_done;          // skip batch elements whose ctl.done is set (slot pool)
};

// Rows of F (and A1, K2) and of the factor e that a stage stages per warp (n <= 128).
template <int N, int STAGE> __host__ __device__ constexpr bool col_rk4_stg() {
  return N <= 128 && STAGE >= COL_RK4_S1 && STAGE <= COL_RK4_S4;
}
template <int N, int STAGE> __host__ __device__ constexpr int col_rk4_nc() {
  return !col_rk4_stg<N, STAGE>() ? 0 : STAGE == COL_RK4_S3 ? 3 : 1;
}
template <int N, int STAGE> __host__ __device__ constexpr int col_rk4_nrl() {
  return (col_rk4_stg<N, STAGE>() && (STAGE == COL_RK4_S1 || STAGE == COL_RK4_S3)) ? 1 : 0;
}

// One warp's column `colid` of a Lawson-RK4 column stage; my_c / my_e are the
// warp's staging rows (col_rk4_nc complex and col_rk4_nrl real rows of M).
// CX > 0 (cluster-resident passes with CX-row tiles): product rows from
// `hrows`, inverse transforms to the cluster's G tiles at `gtile` (null:
// global H / G), as col_tan_body.
template <typename R, int N, int STAGE, int CX = 0>
__device__ __forceinline__ void col_rk4_body(const ColParams<R>& p, int colid, int lane, const cplx<R>* s_tw,
                                             cplx<R>* my_c, R* my_e, const cplx<R>* hrows = nullptr,
                                             cplx<R>* gtile = nullptr) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  const int c = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;   // one warp per (b, ky, channel)

  if (p.use_done && p.ctl[b].done) return;
  const size_t base = ((size_t)(b * 2 + c) * K + ky) * M;
  // The rows of F (and A1, K2, the factor e) that the stage algebra reads,
  // copied into the warp's shared buffers with cp.async before the forward
  // transform, so that their latency overlaps it (n <= 128).
  constexpr bool STG = col_rk4_stg<N, STAGE>();
  constexpr int NC = col_rk4_nc<N, STAGE>();     // F (A1, K2)
  constexpr int NRL = col_rk4_nrl<N, STAGE>();   // e
  if constexpr (STG) {
    for (int s2 = lane; s2 < M; s2 += 32) {
      cp_async_v(my_c + s2, p.F + base + s2);
      if constexpr (NC == 3) { cp_async_v(my_c + M + s2, p.A1 + base + s2); cp_async_v(my_c + 2 * M + s2, p.K2 + base + s2); }
      if constexpr (NRL == 1) cp_async_v(my_e + s2, p.Etab + base + s2);
    }
  }
  cplx<R> r[E];
  if (STAGE != COL_START) {
    if (CX > 0 && hrows) col_rhs_rows<R, N>(hrows, hrows + N, c, ky, lane, s_tw, r);
    else col_load_rhs<R, N>(p.H, b, c, ky, lane, s_tw, r);
  }
  if constexpr (STG) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
  }
  const R h = (R)p.ctl[b].h;
  cplx<R>* rb = p.rec ? p.rec + (size_t)b * p.rec_bstride : nullptr;
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    x[j] = mk<R>(0, 0);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const bool in_mask = !(kx == 0 && ky == 0);
    cplx<R> v = mk<R>(0, 0);
    if (STAGE != COL_START) {
      v = r[j];                                                        // zero at (0,0)
      if (c == 0 && in_mask) v = cadd(v, p.fhat[ky * M + slot]);       // mask * rfft2(forcing)
    }
    const size_t i = base + slot;
    const size_t o = ((size_t)c * K + ky) * M + slot;
    auto put = [&](int q, cplx<R> a) { if (rb) rb[q * VEC + o] = a; };
    // the staged (or, without staging, global) operands at this slot
    [[maybe_unused]] const cplx<R> FV =
        STG ? my_c[slot] : ((STAGE >= COL_RK4_S1 && STAGE <= COL_RK4_S4) ? p.F[i] : mk<R>(0, 0));
    [[maybe_unused]] const cplx<R> A1V = NC == 3 ? my_c[M + slot] : (STAGE == COL_RK4_S3 ? p.A1[i] : mk<R>(0, 0));
    [[maybe_unused]] const cplx<R> K2V = NC == 3 ? my_c[2 * M + slot] : (STAGE == COL_RK4_S3 ? p.K2[i] : mk<R>(0, 0));
    [[maybe_unused]] const R EV = NRL == 1 ? my_e[slot] : ((STAGE == COL_RK4_S1 || STAGE == COL_RK4_S3) ? p.Etab[i] : R(0));
    switch (STAGE) {
      case COL_START: x[j] = p.F[i]; break;
      case COL_RK4_S1: {   // k1 = h v(f); f = e f; k1 = e k1; X2 = f + k1/2   (timestepping.py:74-76)
        const R e = EV;
        cplx<R> k1 = cscale(v, h);
        put(Q_F, FV); put(Q_K1, k1);
        const cplx<R> f = cscale_rn(FV, e);
        k1 = cscale_rn(k1, e);
        p.F[i] = f; p.A1[i] = k1;
        x[j] = cadd(f, cscale(k1, R(0.5)));
        put(Q_X2, x[j]);
      } break;
      case COL_RK4_S2: {   // k2 = h v(X2); X3 = f + k2/2   (:76-77)
        const cplx<R> k2 = cscale(v, h);
        p.K2[i] = k2;
        x[j] = cadd(FV, cscale(k2, R(0.5)));
        put(Q_K2, k2); put(Q_X3, x[j]);
      } break;
      case COL_RK4_S3: {   // k3; f,k1,k2,k3 *= e; X4 = f + k3; acc = f + k1/6 + k2/3 + k3/3   (:77-80)
        const R e = EV;
        cplx<R> k3 = cscale(v, h);
        put(Q_K3, k3);
        const cplx<R> f = cscale_rn(FV, e), a = cscale_rn(A1V, e), q2 = cscale_rn(K2V, e);
        k3 = cscale_rn(k3, e);
        x[j] = cadd(f, k3);
        put(Q_X4, x[j]);
        p.F[i] = cadd(cadd(cadd(f, cdiv_k<6>(a)), cdiv_k<3>(q2)), cdiv_k<3>(k3));
      } break;
      case COL_RK4_S4: {   // k4; f = acc + k4/6   (:79-80)
        const cplx<R> k4 = cscale(v, h);
        put(Q_K4, k4);
        const cplx<R> f = cadd(FV, cdiv_k<6>(k4));
        p.F[i] = f;
        x[j] = f;
      } break;
      default: {           // COL_PLAIN: state_vel output (mhd_jax.py:171-173)
        if (p.diss) v = cadd(v, cscale(p.F[i], diss_L<R>(kx, ky, c == 0 ? p.nu : p.eta)));
        p.OUT[i] = v;
      } break;
    }
  }
  if (!p.produce) return;
  if constexpr (CX > 0) {
    if (gtile) {
      cplx<R> wu[E], wv[E];
      col_uv_transform<R, N>(x, ky, lane, s_tw, wu, wv);
      col_uv_to_tiles<R, N, CX>(wu, wv, gtile, c, ky, lane);
      return;
    }
  }
  col_inverse_uv<R, N>(x, p.G, b, c, ky, lane, s_tw);
}

template <typename R, int N, int STAGE>
__global__ void __launch_bounds__(128) k_col_rk4(ColParams<R> p) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int NC = col_rk4_nc<N, STAGE>(), NRL = col_rk4_nrl<N, STAGE>();
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  __shared__ __align__(16) cplx<R> s_rc[(NC > 0 ? NC : 1) * 4 * M];   // 4 warps per CTA
  __shared__ __align__(16) R s_rr[(NRL > 0 ? NRL : 1) * 4 * M];
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  col_rk4_body<R, N, STAGE>(p, colid, lane, s_tw, s_rc + (threadIdx.x >> 5) * NC * M, s_rr + (threadIdx.x >> 5) * NRL * M);
}

// ---------------------------------------------------------------------------
// Row pass of the forward RHS: products in physical space.
// ---------------------------------------------------------------------------

template <typename R>
struct RowParams {
  const cplx<R>* G;   // [B][NG][K][N]
  cplx<R>* H;         // [B][NH][K][N]
  R* phys;            // optional record of u, v, B_x, B_y: phys + b * phys_bstride is [N][NPH][N]
  long phys_bstride;
  const StepCtl* ctl; // per-batch control (done flags) or null
  const cplx<R>* tw;
  R b0x, b0y;
  int B;
};

// Physical-field record of one stage: phys[x][NPH][pos] with pos the warp-FFT
// position order (see fft.cuh), so that readers with the same transform
// structure use identical indexing.
template <typename R, int N>
__device__ __forceinline__ const R* phys_row(const R* base, int x) {
  return base + (size_t)x * NPH * N;
}

// Load a [nf][K][XT] tile of a [B][nf][K][N] array into shared memory with row
// pitch XT+1.  Asynchronous copies (cp.async: global -> shared without a
// register round trip; 16 bytes per complex double, 8 per complex float);
// each thread waits for its own copies before returning, and the caller's
// __syncthreads then makes the whole tile visible.
template <typename R, int N, int XT>
__device__ __forceinline__ void load_tile(cplx<R>* s, const cplx<R>* __restrict__ g, int nfK, int x0) {
  for (int i = threadIdx.x; i < nfK * XT; i += blockDim.x) {
    const int xt = i % XT, r = i / XT;
    cp_async_c<R>(s + r * (XT + 1) + xt, g + (size_t)r * N + x0 + xt);
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}
template <typename R, int N, int XT>
__device__ __forceinline__ void store_tile(cplx<R>* __restrict__ g, const cplx<R>* s, int nfK, int x0) {
  for (int i = threadIdx.x; i < nfK * XT; i += blockDim.x) {
    const int xt = i % XT, r = i / XT;
    g[(size_t)r * N + x0 + xt] = s[r * (XT + 1) + xt];
  }
}

// Full Hermitian spectrum value at position q (natural order) of the packed
// pair A + iB, from half-spectrum rows sA, sB (pitch XT+1, column w).  The ky=0
// entries contribute only their real parts, as irfft does.
template <typename R, int N, int XT>
__device__ __forceinline__ cplx<R> packed_pair(const cplx<R>* sA, const cplx<R>* sB, int q, int w) {
  constexpr int K = (N - 1) / 3 + 1;
  if (q < K) {
    cplx<R> a = sA[q * (XT + 1) + w], bb = sB[q * (XT + 1) + w];
    if (q == 0) { a.y = 0; bb.y = 0; }
    return mk<R>(a.x - bb.y, a.y + bb.x);
  }
  if (q > N - K) {
    const int qq = N - q;
    cplx<R> a = sA[qq * (XT + 1) + w], bb = sB[qq * (XT + 1) + w];
    return mk<R>(a.x + bb.y, bb.x - a.y);
  }
  return mk<R>(0, 0);
}

// Full Hermitian spectrum value at position q of one real field (imaginary
// part of the transform left zero) from its half-spectrum row sA.
template <typename R, int N, int XT>
__device__ __forceinline__ cplx<R> packed_one(const cplx<R>* sA, int q, int w) {
  constexpr int K = (N - 1) / 3 + 1;
  if (q < K) {
    cplx<R> a = sA[q * (XT + 1) + w];
    if (q == 0) a.y = 0;
    return a;
  }
  if (q > N - K) return cconj(sA[(N - q) * (XT + 1) + w]);
  return mk<R>(0, 0);
}

// Half spectrum (ky < K) of a natural-order forward transform W of one real
// field, written to shared row s1.
template <typename R, int N, int XT>
__device__ __forceinline__ void store_one(const cplx<R> (&W)[N / 32], cplx<R>* s1, int w, int lane) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int q = lane + 32 * j;
    if (q < K) s1[q * (XT + 1) + w] = W[j];
  }
}

// Split a natural-order forward transform W of (P1 + i P2) into the half
// spectra of P1 and P2 and write ky < K into shared rows s1, s2.
template <typename R, int N, int XT>
__device__ __forceinline__ void split_store(const cplx<R> (&W)[N / 32], cplx<R>* s1, cplx<R>* s2, int w, int lane) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    cplx<R> t = shfl_c<R>(W[E - 1 - j], (32 - lane) & 31);
    const cplx<R> P = (lane == 0) ? W[(E - j) % E] : t;
    const int q = lane + 32 * j;
    if (q < K) {
      const cplx<R> Wq = W[j];
      s1[q * (XT + 1) + w] = mk<R>((Wq.x + P.x) * R(0.5), (Wq.y - P.y) * R(0.5));
      s2[q * (XT + 1) + w] = mk<R>((Wq.y + P.y) * R(0.5), (P.x - Wq.x) * R(0.5));
    }
  }
}

// Rows x0 .. x0 + XT - 1 of state b, one warp per row (the CTA's XT warps);
// s_G and s_H are the tile buffers (NG and NH rows of K x (XT + 1)).
// CX (cluster-resident passes): s_G holds the tile unless load_g; the H tile
// goes to the column warps' rows at `hcols` unless that is null.
template <typename R, int N, int XT, bool CX = false>
__device__ __forceinline__ void row_rhs_body(const RowParams<R>& p, int b, int x0, const cplx<R>* s_tw, cplx<R>* s_G,
                                             cplx<R>* s_H, bool load_g = true, cplx<R>* hcols = nullptr) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  if (!CX || load_g) load_tile<R, N, XT>(s_G, p.G + (size_t)b * NG * K * N, NG * K, x0);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;

  // pairs (u, v) and (B_x, B_y) without the mean field (mhd_jax.py:140-149)
  cplx<R> uv[E], bb[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int q = lane + 32 * j;
    uv[j] = packed_pair<R, N, XT>(s_G + 0 * K * (XT + 1), s_G + 1 * K * (XT + 1), q, w);
    bb[j] = packed_pair<R, N, XT>(s_G + 2 * K * (XT + 1), s_G + 3 * K * (XT + 1), q, w);
  }
  fft_dif2<R, N, true>(uv, bb, s_tw, lane);
  cplx<R> W[E];
  R* ph = p.phys ? p.phys + (size_t)b * p.phys_bstride + (size_t)(x0 + w) * NPH * N : nullptr;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const R u = uv[j].x, v = uv[j].y;
    const R bx = bb[j].x + p.b0x, by = bb[j].y + p.b0y;
    if (ph) {
      const int e = lane + 32 * j;
      ph[e] = u; ph[N + e] = v; ph[2 * N + e] = bx; ph[3 * N + e] = by;
    }
    W[j] = mk<R>(fpm(u - v, u + v, bx - by, bx + by), fpm(bx, by, u, v));   // (P1, P2)
    bb[j] = mk<R>(fpm(u, by, v, bx), R(0));                                // (P3, 0), mhd_jax.py:163
  }
  fft_dit2<R, N, false>(W, bb, s_tw, lane);
  split_store<R, N, XT>(W, s_H, s_H + K * (XT + 1), w, lane);
  store_one<R, N, XT>(bb, s_H + 2 * K * (XT + 1), w, lane);
  __syncthreads();
  if constexpr (CX) {
    if (hcols) { scatter_h_tile<R, N, XT>(s_H, hcols, x0); return; }
  }
  store_tile<R, N, XT>(p.H + (size_t)b * NH * K * N, s_H, NH * K, x0);
}

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_rhs(RowParams<R> p) {
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_G = s_tw + fft_smem(N, XT);
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  if (p.ctl && p.ctl[b].done) return;   // whole block belongs to one batch element
  row_rhs_body<R, N, XT>(p, b, x0, s_tw, s_G, s_G + NG * K * (XT + 1));
}

// ---------------------------------------------------------------------------
// Boundary transforms between real fields [B][2][N][N] and the box spectrum.
// ---------------------------------------------------------------------------

// Row pass of rfft2 restricted to ky < K: real rows of both channels -> H[B][2][K][N].
template <typename R>
struct RowFwdParams {
  const R* fields;    // [B][2][N][N]
  cplx<R>* H;         // [B][2][K][N]
  const cplx<R>* tw;
  int B;
};

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_to_box(RowFwdParams<R> p) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_H = s_tw + fft_smem(N, XT);
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  load_twiddles<R, N>(s_tw, p.tw);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = x0 + w;
  const R* u0 = p.fields + ((size_t)(b * 2 + 0) * N + x) * N;
  const R* u1 = p.fields + ((size_t)(b * 2 + 1) * N + x) * N;
  cplx<R> W[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int y = spec_pos<N>(lane, j);
    W[j] = mk<R>(u0[y], u1[y]);
  }
  fft_dit<R, N, false>(W, s_tw, lane);
  split_store<R, N, XT>(W, s_H, s_H + K * (XT + 1), w, lane);
  __syncthreads();
  store_tile<R, N, XT>(p.H + (size_t)b * 2 * K * N, s_H, 2 * K, x0);
}

// Column pass of rfft2: H columns -> box spectrum V (raw rfft2 values, no mask).
template <typename R>
struct ColBoxParams {
  const cplx<R>* H;   // [B][nf][K][N]
  cplx<R>* V;         // [B][nf][K][M] with batch stride vstride (elements)
  const cplx<R>* tw;
  long vstride;
  int B, nf;
};

template <typename R, int N>
__global__ void __launch_bounds__(128) k_col_to_box(ColBoxParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  load_twiddles<R, N>(s_tw, p.tw);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (col >= p.B * p.nf * K) return;   // col = (b*nf + f)*K + ky
  const cplx<R>* hin = p.H + (size_t)col * N;
  cplx<R> v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) v[j] = hin[lane + 32 * j];
  fft_dif<R, N, false>(v, s_tw, lane);
  const int b = col / (p.nf * K), fk = col - b * p.nf * K;
  cplx<R>* vout = p.V + (size_t)b * p.vstride + (size_t)fk * M;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot >= 0) vout[slot] = v[j];
  }
}

// Symmetry group action applied to a box spectrum value at (kx, ky) of channel c
// (reference: symmetry.shift_x / shift_reflect / rot180, jax_scripts/lib/symmetry.py:4-25).
// The source value must be read at kx_src = odd_ny ? -kx : kx.
struct SymOp {
  double sx;   // x shift
  double sy;   // y shift = ny * 2 pi / 8
  int odd;     // ny odd: reflect x and negate
  int rot;     // rot180: conj, channel signs [1, -1]
};

template <typename R>
__device__ __forceinline__ cplx<R> apply_sym(cplx<R> g, int kx_src, int ky, int c, const SymOp& s) {
  // masked wavenumbers: (0,0) is masked out, so both phases are 1 there
  const bool m = !(kx_src == 0 && ky == 0);
  double sn, cs;
  sincos(m ? (double)kx_src * s.sx : 0.0, &sn, &cs);
  cplx<R> a = cmul(mk<R>((R)cs, (R)sn), g);
  sincos(m ? (double)ky * s.sy : 0.0, &sn, &cs);   // ky is unchanged by the x reflection
  a = cmul(mk<R>((R)cs, (R)sn), a);
  if (s.odd) { a.x = -a.x; a.y = -a.y; }
  if (s.rot) { a.y = -a.y; if (c == 1) { a.x = -a.x; a.y = -a.y; } }
  return a;
}

// Column inverse from a box spectrum (2 channels) -> G2[B][2][K][N], with an
// optional symmetry action, optional scaling and optional multiplier (i kx).
template <typename R>
struct ColFromBoxParams {
  const cplx<R>* V;   // [B][2][K][M]
  cplx<R>* G;         // [B][2][K][N]
  const cplx<R>* tw;
  const double* sx;   // [B] or null
  int sx_shared;      // sx[0] applies to every batch element
  double sy;
  int odd, rot, use_sym;
  int mult_ikx;       // multiply by i kx (masked) before the inverse
  int B;
};

template <typename R, int N>
__global__ void __launch_bounds__(128) k_col_from_box(ColFromBoxParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  load_twiddles<R, N>(s_tw, p.tw);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (col >= p.B * 2 * K) return;   // col = (b*2 + c)*K + ky
  const int ky = col % K, bc = col / K, c = bc & 1, b = bc >> 1;
  const cplx<R>* vin = p.V + (size_t)col * M;
  SymOp so; so.sx = p.sx ? p.sx[p.sx_shared ? 0 : b] : 0.0; so.sy = p.sy; so.odd = p.odd; so.rot = p.rot;
  const R inv_n2 = R(1) / (R(N) * R(N));
  cplx<R> v[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int pos = spec_pos<N>(lane, j);
    const int slot = pos_to_slot(pos, N, KMAX, M);
    v[j] = mk<R>(0, 0);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    cplx<R> val;
    if (p.use_sym) {
      const int ksrc = so.odd ? -kx : kx;
      const int ssrc = ksrc >= 0 ? ksrc : ksrc + M;
      val = apply_sym<R>(vin[ssrc], ksrc, ky, c, so);
    } else {
      val = vin[slot];
    }
    if (p.mult_ikx) val = cimul(val, (kx == 0 && ky == 0) ? R(0) : (R)kx);
    v[j] = cscale(val, inv_n2);
  }
  fft_dit<R, N, true>(v, s_tw, lane);
  cplx<R>* gout = p.G + (size_t)col * N;
#pragma unroll
  for (int j = 0; j < E; ++j) gout[lane + 32 * j] = v[j];
}

// Row c2r of the two channels G2[B][2][K][N] -> real fields.
//   mode 0: out = u
//   mode 1: out = base - u   (objective residual irfft2(f0 - f) with irfft2(f0) = base)
//   mode 2: out = base + u
// Optionally accumulates per-row sums of out^2 (loss) into rowsq[B][N].
template <typename R>
struct RowFromBoxParams {
  const cplx<R>* G;   // [B][2][K][N]
  R* out;             // [B][2][N][N]
  const R* base;      // [B][2][N][N] or null
  double* rowsq;      // [B][N] or null
  const cplx<R>* tw;
  int B, mode;
};

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_from_box(RowFromBoxParams<R> p) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_G = s_tw + fft_smem(N, XT);
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  load_twiddles<R, N>(s_tw, p.tw);
  load_tile<R, N, XT>(s_G, p.G + (size_t)b * 2 * K * N, 2 * K, x0);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = x0 + w;
  cplx<R> z[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int q = spec_pos<N>(lane, j);
    z[j] = packed_pair<R, N, XT>(s_G, s_G + K * (XT + 1), q, w);
  }
  fft_dit<R, N, true>(z, s_tw, lane);
  R* o0 = p.out + ((size_t)(b * 2 + 0) * N + x) * N;
  R* o1 = p.out + ((size_t)(b * 2 + 1) * N + x) * N;
  const R* b0 = p.base ? p.base + ((size_t)(b * 2 + 0) * N + x) * N : nullptr;
  const R* b1 = p.base ? p.base + ((size_t)(b * 2 + 1) * N + x) * N : nullptr;
  double sq = 0.0;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int y = lane + 32 * j;
    R a = z[j].x, c = z[j].y;
    if (p.mode == 1) { a = b0[y] - a; c = b1[y] - c; }
    else if (p.mode == 2) { a = b0[y] + a; c = b1[y] + c; }
    o0[y] = a; o1[y] = c;
    sq += (double)a * (double)a + (double)c * (double)c;
  }
  if (p.rowsq) {
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if (lane == 0) p.rowsq[(size_t)b * N + x] = sq;
  }
}

// ---------------------------------------------------------------------------
// Small elementwise kernels
// ---------------------------------------------------------------------------

// Full rfft2 layout [B][2][N][N/2+1] <-> box [B][2][K][M].
template <typename R>
__global__ void k_gather_box(const cplx<R>* full, cplx<R>* box, int n, int B) {
  const Geom g = make_geom(n);
  const int nh = n / 2 + 1;
  const long total = (long)B * 2 * g.K * g.M;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int slot = i % g.M; const long r = i / g.M; const int ky = r % g.K; const long bc = r / g.K;
    const int kx = slot_to_kx(slot, g.kmax, g.M);
    const int pos = kx >= 0 ? kx : kx + n;
    box[i] = full[(bc * n + pos) * nh + ky];
  }
}

template <typename R>
__global__ void k_scatter_box(const cplx<R>* box, cplx<R>* full, int n, int B) {
  const Geom g = make_geom(n);
  const int nh = n / 2 + 1;
  const long total = (long)B * 2 * n * nh;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int ky = i % nh; const long r = i / nh; const int pos = r % n; const long bc = r / n;
    const int slot = (ky < g.K) ? pos_to_slot(pos, n, g.kmax, g.M) : -1;
    full[i] = slot >= 0 ? box[(bc * g.K + ky) * g.M + slot] : mk<R>(0, 0);
  }
}

// Lawson-RK4 setup: h = (T/nc)/ms and e = exp(h/2 L) * mask per batch element.
template <typename R>
__global__ void k_rk4_setup(const double* T, int nc, int ms, StepCtl* ctl, R* Etab, int n, double nu, double eta, int B) {
  const Geom g = make_geom(n);
  const long per = 2L * g.K * g.M;
  const long total = (long)B * per;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / per);
    const double tseg = T[b] / (double)nc;          // loss_functions.py:63 T/num_checkpoints
    const R h = (R)(tseg / (double)ms);              // timestepping.py:69 h = t/steps
    if (i % per == 0) { ctl[b].t = tseg; ctl[b].h = (double)h; }
    const int slot = i % g.M; const long r = i / g.M; const int ky = r % g.K; const int c = (r / g.K) & 1;
    const int kx = slot_to_kx(slot, g.kmax, g.M);
    const R L = diss_L<R>(kx, ky, (R)(c == 0 ? nu : eta));
    const bool msk = !(kx == 0 && ky == 0);
    Etab[i] = msk ? exp(h / R(2) * L) : R(0);        // timestepping.py:70-72
  }
}

// out -= P_sym(rest): the symmetry action on modes outside the box, which in
// real space is x -> -x with negation (odd ny) and a 180 degree rotation with
// channel signs [1, -1] (rot); shift_x and the y-phase of shift_reflect use
// masked wavenumbers and leave these modes unchanged (symmetry.py:4-25).
template <typename R>
__global__ void k_sub_sym_phys(R* out, const R* rest, int odd, int rot, int n, int B) {
  const long total = (long)B * 2 * n * n;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int y = i % n; const long r = i / n; const int x = r % n; const long bc = r / n; const int c = bc & 1;
    const int sx = (odd ? -1 : 1) * (rot ? -1 : 1), sy = rot ? -1 : 1;
    const int xs = ((sx * x) % n + n) % n, ys = ((sy * y) % n + n) % n;
    R f = rest[(bc * n + xs) * n + ys];
    if (odd) f = -f;
    if (rot && c == 1) f = -f;
    out[i] -= f;
  }
}

// Per-row sums of squares of real fields [B][2][N][N]: rowsq[b][x] (one warp per (b, x)).
template <typename R>
__global__ void k_rowsq(const R* f, double* rowsq, int n) {
  const int bx = blockIdx.x, b = bx / n, x = bx % n;
  double s = 0.0;
  for (int c = 0; c < 2; ++c) {
    const R* row = f + ((size_t)(b * 2 + c) * n + x) * n;
    for (int y = threadIdx.x; y < n; y += 32) s += (double)row[y] * (double)row[y];
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) rowsq[bx] = s;
}

template <typename R>
__global__ void k_axpy(R* y, const R* x, R a, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) y[i] += a * x[i];
}

// Slot pool: initialise one slot's control (steps_total = 0 marks it inactive).
static __global__ void k_pool_init(StepCtl* ctl, int first, int count, int steps_total) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  StepCtl& c = ctl[first + i];
  c.steps_total = steps_total; c.steps_done = 0; c.done = steps_total > 0 ? 0 : 1;
  c.attempts = 0; c.accepted = 0; c.rejected = 0; c.pending_accept = 0;
}

// Slot pool: count one finished step per active slot; a slot whose budget is
// spent is marked done and skipped by every later launch.
static __global__ void k_pool_count(StepCtl* ctl, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  StepCtl& c = ctl[b];
  if (c.done || c.steps_total <= 0) return;
  c.steps_done += 1;
  if (c.steps_done >= c.steps_total) c.done = 1;
}

// Deterministic per-batch reduction of row partials: out[b] = scale * sum_x rowsq[b][x].
static __global__ void k_reduce_rows(const double* rowsq, double* out, int n, int B, double scale) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  double s = 0.0;
  for (int x = 0; x < n; ++x) s += rowsq[(size_t)b * n + x];
  out[b] = s * scale;
}

}  // namespace ecs
