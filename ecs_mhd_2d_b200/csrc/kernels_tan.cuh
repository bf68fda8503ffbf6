// Tangent (forward-mode) kernels of the shooting map: the JVP used as the
// Newton-GMRES matvec (reference: jax.jvp of objective_RPO, jax_scripts/lib/utils.py:108).
//
// A batch of B tangents shares one primal trajectory.  The primal solve records,
// per step (Lawson-RK4) or attempt (Lawson-RK4(3)), the compact stage inputs and
// stage derivatives; the tangent pass regenerates the primal's 4 physical
// fields (u, v, B_x, B_y) for a chunk of stages in one batched launch pair
// (shared by all tangents) and then advances the tangents with the linearised
// products of the Basdevant form (see kernels.cuh)
//   dP1 = 2 (u du - v dv) - 2 (B_x dB_x - B_y dB_y)
//   dP2 = B_x dB_y + B_y dB_x - u dv - v du
//   dP3 = u dB_y + B_y du - v dB_x - B_x dv
// and the product rule through the integrating factor, e' = e L h'/2.
#pragma once

#include "kernels.cuh"
#include "kernels_rk43.cuh"

namespace ecs {


// ---------------------------------------------------------------------------
// Regeneration of primal physical fields for a list of recorded stage inputs.
// ---------------------------------------------------------------------------
template <typename R>
struct ColRegenParams {
  const cplx<R>* rec;     // record base
  const long* items;      // [nitems] offsets (in box vectors) of the stage inputs in rec
  cplx<R>* G;             // [nitems][NG][K][N]
  const cplx<R>* tw;
  int nitems;
};

template <typename R, int N>
__global__ void __launch_bounds__(128) k_col_regen(ColRegenParams<R> p) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  load_twiddles<R, N>(s_tw, p.tw);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int col = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (col >= p.nitems * K * 2) return;
  const int ch = col & 1, ik = col >> 1, it = ik / K, ky = ik - it * K;   // one warp per (item, ky, channel)
  const cplx<R>* y = p.rec + (size_t)p.items[it] * VEC + (size_t)(ch * K + ky) * M;
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    x[j] = slot >= 0 ? y[slot] : mk<R>(0, 0);
  }
  col_inverse_uv<R, N>(x, p.G, it, ch, ky, lane, s_tw);
}

// Physical fields of each item: Phys[it][x][NPH][pos] (B_x, B_y include b0).
template <typename R>
struct RowPhysParams {
  const cplx<R>* G;   // [nitems][NG][K][N]
  R* phys;            // [nitems][N][NPH][N]
  const cplx<R>* tw;
  R b0x, b0y;
  int nitems;
};

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_phys(RowPhysParams<R> p) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_G = s_tw + fft_smem(N, XT);
  const int tiles = N / XT;
  const int it = blockIdx.x / tiles, x0 = (blockIdx.x - it * tiles) * XT;
  load_twiddles<R, N>(s_tw, p.tw);
  load_tile<R, N, XT>(s_G, p.G + (size_t)it * NG * K * N, NG * K, x0);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = x0 + w;
  R* ph = p.phys + (((size_t)it * N + x) * NPH) * N;
  cplx<R> uv[E], bb[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    uv[j] = packed_pair<R, N, XT>(s_G, s_G + K * (XT + 1), lane + 32 * j, w);
    bb[j] = packed_pair<R, N, XT>(s_G + 2 * K * (XT + 1), s_G + 3 * K * (XT + 1), lane + 32 * j, w);
  }
  fft_dif2<R, N, true>(uv, bb, s_tw, lane);
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int e = lane + 32 * j;
    ph[e] = uv[j].x; ph[N + e] = uv[j].y;
    ph[2 * N + e] = bb[j].x + p.b0x; ph[3 * N + e] = bb[j].y + p.b0y;   // B carries the mean field (mhd_jax.py:145-149)
  }
}

// ---------------------------------------------------------------------------
// Tangent row pass: linearised products around the primal physical fields.
// ---------------------------------------------------------------------------
template <typename R>
struct RowTanParams {
  const cplx<R>* G;     // tangent [B][NG][K][N]
  cplx<R>* H;           // tangent [B][NH][K][N]
  const R* phys;        // primal physical fields of this stage: phys + b * phys_bstride is [N][NPH][N]
  long phys_bstride;    // 0: one primal shared by the batch
  const cplx<R>* tw;
  const StepCtl* ctl;   // optional per-candidate control: batch elements whose ctl.done is set are skipped
  int B;
};

// The linearised products of one row in physical space (dP1, dP2 in duv, dP3 in dbb).
template <typename R, int E>
__device__ __forceinline__ void row_tan_products(cplx<R> (&duv)[E], cplx<R> (&dbb)[E], const R (&pu)[E],
                                                 const R (&pv)[E], const R (&pbx)[E], const R (&pby)[E]) {
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const R du = duv[j].x, dv = duv[j].y, dbx = dbb[j].x, dby = dbb[j].y;
    const R u = pu[j], v = pv[j], bx = pbx[j], by = pby[j];
    duv[j] = mk<R>(R(2) * (fpm(u, du, v, dv) - fpm(bx, dbx, by, dby)),     // dP1
                   fpp(bx, dby, by, dbx) - fpp(u, dv, v, du));              // dP2
    dbb[j] = mk<R>(fpp(u, dby, by, du) - fpp(v, dbx, bx, dv), R(0));        // dP3
  }
}

// Rows x0 .. x0 + XT - 1 of tangent b, one warp per row (the CTA's XT warps);
// s_G and s_H are the tile buffers (NG and NH rows of K x (XT + 1)).
// CX (cluster-resident passes): s_G already holds the tile (written
// by the column pass) unless load_g, and the H tile goes to the column warps'
// rows at `hcols` (scatter_h_tile) unless that is null (global H).
template <typename R, int N, int XT, bool CX = false>
__device__ __forceinline__ void row_tan_body(const RowTanParams<R>& p, int b, int x0, const cplx<R>* s_tw,
                                             cplx<R>* s_G, cplx<R>* s_H, bool load_g = true,
                                             cplx<R>* hcols = nullptr) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int x = x0 + w;
  // primal u, v, B_x, B_y of this row, loaded first so that the loads overlap
  // the tile load and the inverse transforms (n <= 128); at n = 256 they would
  // hold 4 E = 32 registers across the transform, so they are loaded after it
  const R* ph = phys_row<R, N>(p.phys + (size_t)b * p.phys_bstride, x);
  R pu[E], pv[E], pbx[E], pby[E];
  auto load_phys = [&]() {
#pragma unroll
    for (int j = 0; j < E; ++j) {
      const int e = lane + 32 * j;
      pu[j] = ph[e]; pv[j] = ph[N + e]; pbx[j] = ph[2 * N + e]; pby[j] = ph[3 * N + e];
    }
  };
  if constexpr (N <= 128) load_phys();
  if (!CX || load_g) load_tile<R, N, XT>(s_G, p.G + (size_t)b * NG * K * N, NG * K, x0);
  __syncthreads();
  cplx<R> duv[E], dbb[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const int q = lane + 32 * j;
    duv[j] = packed_pair<R, N, XT>(s_G + 0 * K * (XT + 1), s_G + 1 * K * (XT + 1), q, w);
    dbb[j] = packed_pair<R, N, XT>(s_G + 2 * K * (XT + 1), s_G + 3 * K * (XT + 1), q, w);
  }
  fft_dif2<R, N, true>(duv, dbb, s_tw, lane);
  if constexpr (N > 128) load_phys();
  row_tan_products<R, E>(duv, dbb, pu, pv, pbx, pby);
  fft_dit2<R, N, false>(duv, dbb, s_tw, lane);
  split_store<R, N, XT>(duv, s_H, s_H + K * (XT + 1), w, lane);
  store_one<R, N, XT>(dbb, s_H + 2 * K * (XT + 1), w, lane);
  __syncthreads();
  if constexpr (CX) {
    if (hcols) { scatter_h_tile<R, N, XT>(s_H, hcols, x0); return; }
  }
  store_tile<R, N, XT>(p.H + (size_t)b * NH * K * N, s_H, NH * K, x0);
}

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32, 2) k_row_tan(RowTanParams<R> p) {
  constexpr int K = (N - 1) / 3 + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_G = s_tw + fft_smem(N, XT);
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  if (p.ctl && p.ctl[b].done) return;   // the whole CTA belongs to batch element b
  row_tan_body<R, N, XT>(p, b, x0, s_tw, s_G, s_G + NG * K * (XT + 1));
}

// ---------------------------------------------------------------------------
// Tangent column pass: forward transform of the linearised products and the
// tangent of the stepper algebra.
// ---------------------------------------------------------------------------
enum TanStage : int {
  TS_START = 0,                  // inverse transforms of the tangent state (dF / dX0)
  T4_S1 = 1, T4_S2, T4_S3, T4_S4,   // Lawson-RK4 stages
  T43_INIT = 10, T43_A, T43_B, T43_C, T43_D, T43_E,   // Lawson-RK4(3) stages
  T43_START = 16,                // inverse transforms of dX0 (before T43_INIT)
  T43_EA = 17,                   // T43_E of an attempt, then T43_A of the next (accepted) attempt, one launch
};
// Tangent slots (Lawson-RK4 uses the first three).
enum TanSlot { D_F = 0, D_A1, D_K2, D_NS4 = 3 };

template <typename R>
struct ColTanParams {
  const cplx<R>* H;     // [B][NH][K][N]
  cplx<R>* G;           // [B][NG][K][N]
  cplx<R>* D;           // tangent slots [B][nslot][2][K][M]
  int nslot;
  const cplx<R>* rec;   // primal record of this step/attempt
  const double* dT;     // [B]
  double t, h;          // Lawson-RK4: t unused; Lawson-RK4(3): t = T, h = attempt step
  double dscale;        // Lawson-RK4: dh = dT * dscale; Lawson-RK4(3): dt = dT * dscale
  const cplx<R>* tw;
  R nu, eta;
  int B, stage, produce;
  // Several candidates, one tangent each (ecs_jvp_multi; Lawson-RK4 stages):
  // ctl[b] gives candidate b's step size h and done flag (skipped once done),
  // rec + b * rec_bstride its record, dscale_b[b] its dT scale, and
  // etab + b * 2 K M its factor exp(h/2 L) mask.  All null/0 for one candidate.
  const StepCtl* ctl;
  long rec_bstride;
  const double* dscale_b;
  const R* etab;
  const cplx<R>* rec2;  // T43_EA: the next attempt's record (h is the next attempt's step)
};

// Record vectors (bits of Rk43Rec) and tangent slots (bits of Rk43Slot) that the
// stage algebra of an adaptive stage reads; they are staged per column into
// shared memory at the start (see k_col_tan).
__host__ __device__ constexpr unsigned tan_qmask(int stage) {
  return stage == T43_INIT ? (1u << RR_K1)
       : stage == T43_A ? (1u << RR_X0) | (1u << RR_K1) | (1u << RR_E)
       : stage == T43_B ? (1u << RR_K2)
       : stage == T43_C ? (1u << RR_X0) | (1u << RR_K1) | (1u << RR_K2) | (1u << RR_K3) | (1u << RR_E)
       : stage == T43_D ? (1u << RR_K4)
       : stage == T43_E || stage == T43_EA ? (1u << RR_K5) : 0u;
}
// Record vectors of the next attempt read by T43_EA (from rec2).
__host__ __device__ constexpr unsigned tan_qmask2(int stage) {
  return stage == T43_EA ? (1u << RR_X0) | (1u << RR_K1) | (1u << RR_E) : 0u;
}
__host__ __device__ constexpr unsigned tan_dmask(int stage) {
  return stage == T43_START ? (1u << S_X0)
       : stage == T43_A ? (1u << S_X0) | (1u << S_K1)
       : stage == T43_B ? (1u << S_XE)
       : stage == T43_C ? (1u << S_XE) | (1u << S_K1E) | (1u << S_K2)
       : stage == T43_D ? (1u << S_K1) | (1u << S_K2) | (1u << S_K3) | (1u << S_X2)
       : stage == T43_E || stage == T43_EA ? (1u << S_XF) : 0u;
}
__host__ __device__ constexpr int popc_c(unsigned m) { return m ? (int)(m & 1u) + popc_c(m >> 1) : 0; }

// Operand rows staged per warp by a tangent column stage (shared memory, M entries each).
template <int N, int STAGE> __host__ __device__ constexpr int col_tan_nop() {
  return N <= 128 ? popc_c(tan_qmask(STAGE)) + popc_c(tan_qmask2(STAGE)) + popc_c(tan_dmask(STAGE)) : 0;
}

// One warp's column `colid` of a tangent column stage; `my_op` is the warp's
// staging buffer (col_tan_nop rows of M entries), `s_tw` the twiddle image.
// CX > 0 (cluster-resident passes with CX-row tiles): the product rows come from
// `hrows` (the warp's rows in shared memory, see scatter_h_tile) and the
// inverse transforms go to the cluster's G tiles at `gtile` (col_uv_to_tiles);
// a null pointer selects global H / G instead.
// DSH (cluster-resident adaptive passes): the tangent slots of this column live
// in shared memory at `dsh` ([S_NSLOT][M]) instead of global D.
template <typename R, int N, int STAGE, int CX = 0, bool DSH = false>
__device__ __forceinline__ void col_tan_body(const ColTanParams<R>& p, int colid, int lane, const cplx<R>* s_tw,
                                             cplx<R>* my_op, const cplx<R>* hrows = nullptr,
                                             cplx<R>* gtile = nullptr, cplx<R>* dsh = nullptr) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  const int ch = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;   // one warp per (b, ky, channel)
  if (p.ctl && p.ctl[b].done) return;
  cplx<R>* D = p.D + (size_t)b * p.nslot * VEC;
  const cplx<R>* Q = p.rec + (size_t)b * p.rec_bstride;
  constexpr bool rk43 = STAGE >= T43_INIT;
  constexpr bool has_rhs = !(STAGE == TS_START || STAGE == T43_A || STAGE == T43_START);
  const R h = p.ctl ? (R)p.ctl[b].h : (R)p.h, t = (R)p.t;
  const R dpar = (R)(p.dT[b] * (p.dscale_b ? p.dscale_b[b] : p.dscale));   // dh (RK4) or dt (RK4(3))
  // The record vectors and tangent slots the stage algebra reads, this column's
  // rows of them (M entries each), copied into the warp's shared buffer with
  // cp.async before the forward transform, so that their latency overlaps it
  // without holding registers (adaptive stages, n <= 128: static shared memory).
  constexpr unsigned QM = N <= 128 ? tan_qmask(STAGE) : 0u, DM = (N <= 128 && !DSH) ? tan_dmask(STAGE) : 0u;
  constexpr unsigned QM2 = N <= 128 ? tan_qmask2(STAGE) : 0u;
  constexpr int NQ = popc_c(QM), NQ2 = popc_c(QM2), NOP = NQ + NQ2 + popc_c(DM);
  const cplx<R>* Q2 = p.rec2;
  if constexpr (NOP > 0) {
    const size_t row = ((size_t)ch * K + ky) * M;
    int v = 0;
#pragma unroll
    for (int bit = 0; bit < 16; ++bit) {
      if ((QM >> bit) & 1u) {
        for (int s2 = lane; s2 < M; s2 += 32) cp_async_c<R>(my_op + v * M + s2, Q + bit * VEC + row + s2);
        ++v;
      }
    }
#pragma unroll
    for (int bit = 0; bit < 16; ++bit) {
      if ((QM2 >> bit) & 1u) {
        for (int s2 = lane; s2 < M; s2 += 32) cp_async_c<R>(my_op + v * M + s2, Q2 + bit * VEC + row + s2);
        ++v;
      }
    }
#pragma unroll
    for (int bit = 0; bit < 16; ++bit) {
      if ((DM >> bit) & 1u) {
        for (int s2 = lane; s2 < M; s2 += 32) cp_async_c<R>(my_op + v * M + s2, D + bit * VEC + row + s2);
        ++v;
      }
    }
  }
  cplx<R> r[E];
  if (has_rhs) {
    if (CX > 0 && hrows) col_rhs_rows<R, N>(hrows, hrows + N, ch, ky, lane, s_tw, r);
    else col_load_rhs<R, N>(p.H, b, ch, ky, lane, s_tw, r);
  }
  if constexpr (NOP > 0) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
  }
  const R coeff = ch == 0 ? p.nu : p.eta;
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    x[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    const bool in_mask = !(kx == 0 && ky == 0);
    cplx<R> dv = mk<R>(0, 0);
    if (has_rhs) dv = r[j];                              // the tangent has no forcing
    const size_t o = ((size_t)ch * K + ky) * M + slot;
    const R L = diss_L<R>(kx, ky, coeff);
    cplx<R> xin = mk<R>(0, 0);
    if (!rk43) {
      // Lawson-RK4: e = exp(h/2 L) mask, de = e L dh/2; dk = dh v + h dv with v = k/h
      const R e = p.etab ? p.etab[(size_t)b * VEC + o] : in_mask ? exp(h / R(2) * L) : R(0);
      const R de = e * L * (dpar / R(2));
      auto dk_of = [&](int q) { return lin2_rn(Q[q * VEC + o], dpar / h, dv, h); };
      switch (STAGE) {
        case TS_START: xin = D[D_F * VEC + o]; break;
        case T4_S1: {
          const cplx<R> dk1 = dk_of(Q_K1);
          const cplx<R> df1 = lin2_rn(Q[Q_F * VEC + o], de, D[D_F * VEC + o], e);
          const cplx<R> da1 = lin2_rn(Q[Q_K1 * VEC + o], de, dk1, e);
          D[D_F * VEC + o] = df1; D[D_A1 * VEC + o] = da1;
          xin = cadd(df1, cscale(da1, R(0.5)));
        } break;
        case T4_S2: {
          const cplx<R> dk2 = dk_of(Q_K2);
          D[D_K2 * VEC + o] = dk2;
          xin = cadd(D[D_F * VEC + o], cscale(dk2, R(0.5)));
        } break;
        case T4_S3: {
          const cplx<R> dk3 = dk_of(Q_K3);
          const cplx<R> f1 = cscale_rn(Q[Q_F * VEC + o], e), a1 = cscale_rn(Q[Q_K1 * VEC + o], e);
          const cplx<R> df2 = lin2_rn(f1, de, D[D_F * VEC + o], e);
          const cplx<R> db1 = lin2_rn(a1, de, D[D_A1 * VEC + o], e);
          const cplx<R> db2 = lin2_rn(Q[Q_K2 * VEC + o], de, D[D_K2 * VEC + o], e);
          const cplx<R> db3 = lin2_rn(Q[Q_K3 * VEC + o], de, dk3, e);
          xin = cadd(df2, db3);
          D[D_F * VEC + o] = cadd(cadd(cadd(df2, cdiv_k<6>(db1)), cdiv_k<3>(db2)), cdiv_k<3>(db3));
        } break;
        default: {   // T4_S4
          const cplx<R> dk4 = dk_of(Q_K4);
          xin = cadd(D[D_F * VEC + o], cdiv_k<6>(dk4));
          D[D_F * VEC + o] = xin;
        } break;
      }
    } else {
      // Lawson-RK4(3): e = exp(t L h/2), de = e L h/2 dt; dk = dt v + t dv with v = k/t
      // staged operands (shared memory) or, without staging, global memory
      auto QV = [&](int q) -> cplx<R> {
        if constexpr (NOP > 0) return my_op[popc_c(QM & ((1u << q) - 1u)) * M + slot];
        else return Q[q * VEC + o];
      };
      // (e, e L h/2) of this attempt from the primal record (stages A and C use them)
      const cplx<R> eg = (STAGE == T43_A || STAGE == T43_C) ? QV(RR_E) : mk<R>(0, 0);
      [[maybe_unused]] const R e = eg.x;
      [[maybe_unused]] const R de = eg.y * dpar;
      auto Q2V = [&](int q) -> cplx<R> {
        if constexpr (NOP > 0) return my_op[(NQ + popc_c(QM2 & ((1u << q) - 1u))) * M + slot];
        else return Q2[q * VEC + o];
      };
      auto DV = [&](int d) -> cplx<R> {
        if constexpr (DSH) return dsh[d * M + slot];
        else if constexpr (NOP > 0) return my_op[(NQ + NQ2 + popc_c(DM & ((1u << d) - 1u))) * M + slot];
        else return D[d * VEC + o];
      };
      auto DW = [&](int d, cplx<R> v) {
        if constexpr (DSH) dsh[d * M + slot] = v;
        else D[d * VEC + o] = v;
      };
      auto dk_of = [&](int q) { return lin2_rn(QV(q), dpar / t, dv, t); };
      // the A and E algebra, written with explicitly rounded operations: the
      // merged pass T43_EA computes exactly what T43_E followed by T43_A does
      auto stage_e = [&]() { return lin2_rn(QV(RR_K5), dpar / t, dv, t); };   // dk5
      auto stage_a = [&](cplx<R> x0, cplx<R> k1, cplx<R> eg_, cplx<R> dx0, cplx<R> dk1, R h_) {
        const R e_ = eg_.x, de_ = mul_rn(eg_.y, dpar);
        const cplx<R> dxe = lin2_rn(x0, de_, dx0, e_), dk1e = lin2_rn(k1, de_, dk1, e_);
        DW(S_XE, dxe); DW(S_K1E, dk1e);
        cplx<R> half = cscale(dk1e, h_);
        half.x = mul_rn(half.x, R(0.5)); half.y = mul_rn(half.y, R(0.5));
        return mk<R>(add_rn(dxe.x, half.x), add_rn(dxe.y, half.y));
      };
      switch (STAGE) {
        case T43_START: xin = DV(S_X0); break;
        case T43_INIT: DW(S_K1, dk_of(RR_K1)); break;
        case T43_A: xin = stage_a(QV(RR_X0), QV(RR_K1), eg, DV(S_X0), DV(S_K1), h); break;
        case T43_B: {
          const cplx<R> dk2 = dk_of(RR_K2);
          DW(S_K2, dk2);
          xin = cadd(DV(S_XE), cscale(cscale(dk2, h), R(0.5)));
        } break;
        case T43_C: {
          const cplx<R> dk3 = dk_of(RR_K3);
          const cplx<R> xe = cscale_rn(QV(RR_X0), e), k1e = cscale_rn(QV(RR_K1), e);
          const cplx<R> dx2 = lin2_rn(xe, de, DV(S_XE), e);
          const cplx<R> dk1ee = lin2_rn(k1e, de, DV(S_K1E), e);
          const cplx<R> dk2e = lin2_rn(QV(RR_K2), de, DV(S_K2), e);
          const cplx<R> dk3e = lin2_rn(QV(RR_K3), de, dk3, e);
          DW(S_X2, dx2); DW(S_K1, dk1ee); DW(S_K2, dk2e); DW(S_K3, dk3e);
          xin = cadd_scaled_rn(dx2, dk3e, h);
        } break;
        case T43_D: {
          const cplx<R> dk4 = dk_of(RR_K4);
          const cplx<R> acc = cadd(cadd(cadd(cdiv_k<6>(DV(S_K1)), cdiv_k<3>(DV(S_K2))),
                                        cdiv_k<3>(DV(S_K3))), cdiv_k<6>(dk4));
          xin = cadd_scaled_rn(DV(S_X2), acc, h);
          DW(S_XF, xin);
        } break;
        case T43_E: {   // accepted attempt, promote (dxf, dk5) -> (dx0, dk1)
          DW(S_K1, stage_e());
          DW(S_X0, DV(S_XF));
        } break;
        default: {      // T43_EA: T43_E, then T43_A of the next attempt on the promoted values
          const cplx<R> dk1 = stage_e(), dx0 = DV(S_XF);
          DW(S_K1, dk1);
          DW(S_X0, dx0);
          xin = stage_a(Q2V(RR_X0), Q2V(RR_K1), Q2V(RR_E), dx0, dk1, h);
        } break;
      }
    }
    x[j] = xin;
  }
  if (!p.produce || STAGE == T43_INIT || STAGE == T43_E) return;
  if constexpr (CX > 0) {
    if (gtile) {
      cplx<R> wu[E], wv[E];
      col_uv_transform<R, N>(x, ky, lane, s_tw, wu, wv);
      col_uv_to_tiles<R, N, CX>(wu, wv, gtile, ch, ky, lane);
      return;
    }
  }
  col_inverse_uv<R, N>(x, p.G, b, ch, ky, lane, s_tw);
}

template <typename R, int N, int STAGE>
__global__ void __launch_bounds__(128) k_col_tan(ColTanParams<R> p) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int NOP = col_tan_nop<N, STAGE>();
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  __shared__ __align__(16) cplx<R> s_op[(NOP > 0 ? NOP : 1) * 4 * M];   // 4 warps per CTA
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  col_tan_body<R, N, STAGE>(p, colid, lane, s_tw, s_op + (threadIdx.x >> 5) * NOP * M);
}

// Rejected Lawson-RK4(3) attempt: the carried k1 becomes e^2 k1 (timestepping.py:267,275,297);
// its tangent is d(e (e k1)) with e' = e L h/2 dt ((e, e L h/2) from the attempt's record).
// The carried dk1 at entry o after a rejected attempt (record rec), dpar = dT * dscale.
template <typename R>
__device__ __forceinline__ cplx<R> tan_reject_k1(const cplx<R>* rec, size_t VEC, size_t o, R dpar, cplx<R> dk1) {
  const cplx<R> eg = rec[RR_E * VEC + o];   // (e, e L h/2) of the attempt
  const R e = eg.x;
  const R de = eg.y * dpar;
  const cplx<R> k1 = rec[RR_K1 * VEC + o];
  const cplx<R> k1e = cscale_rn(k1, e);
  const cplx<R> dk1e = lin2_rn(k1, de, dk1, e);
  return lin2_rn(k1e, de, dk1e, e);
}
// Entry o of tangent Db (slots of one tangent).
template <typename R>
__device__ __forceinline__ void tan_reject_at(cplx<R>* Db, const cplx<R>* rec, size_t VEC, size_t o, R dpar) {
  Db[S_K1 * VEC + o] = tan_reject_k1<R>(rec, VEC, o, dpar, Db[S_K1 * VEC + o]);
}

template <typename R>
__global__ void k_tan_reject(cplx<R>* D, int nslot, const cplx<R>* rec, const double* dT, double dscale, int n,
                             int B) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  const long total = (long)B * VEC;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / VEC);
    const size_t o = i - (size_t)b * VEC;
    tan_reject_at<R>(D + (size_t)b * nslot * VEC, rec, VEC, o, (R)(dT[b] * dscale));
  }
}

// W[b] = dPhi[b] + i kx dsx[b] Phi (the tangent of shift_x before the symmetry
// action, symmetry.py:4-5; kx masked).
template <typename R>
__global__ void k_tan_shift(const cplx<R>* dphi, long dstride, const cplx<R>* phi, const double* dsx, cplx<R>* W,
                            int n, int B) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  const long total = (long)B * VEC;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / VEC);
    const size_t o = i - (size_t)b * VEC;
    const int slot = o % g.M; const int ky = (o / g.M) % g.K;
    const int kx = slot_to_kx(slot, g.kmax, g.M);
    const R kxm = (kx == 0 && ky == 0) ? R(0) : (R)kx;
    W[i] = cadd(dphi[(size_t)b * dstride + o], cimul(cscale(phi[o], (R)dsx[b]), kxm));
  }
}

// Tangents of the phase conditions: dpt = mean(vt * du0), dpx = mean(vx * du0)
// over 2 n^2 entries (loss_functions.py:124-125); one block per tangent.
template <typename R>
__global__ void k_phase_dot(const R* vt, const R* vx, const R* du, double* dpt, double* dpx, int n) {
  const int b = blockIdx.x;
  const long cnt = 2L * n * n;
  const R* d = du + (size_t)b * cnt;
  double st = 0.0, sx = 0.0;
  for (long i = threadIdx.x; i < cnt; i += blockDim.x) { st += (double)vt[i] * d[i]; sx += (double)vx[i] * d[i]; }
  __shared__ double s1[32], s2[32];
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) { st += __shfl_xor_sync(0xffffffffu, st, o); sx += __shfl_xor_sync(0xffffffffu, sx, o); }
  if ((threadIdx.x & 31) == 0) { s1[threadIdx.x >> 5] = st; s2[threadIdx.x >> 5] = sx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, c = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { a += s1[w]; c += s2[w]; }
    dpt[b] = a / (double)cnt; dpx[b] = c / (double)cnt;
  }
}

}  // namespace ecs
