// Cluster-resident tangent sweep of the adaptive Lawson-RK4(3) linearisation:
// one launch runs a whole list of tangent passes (the column stages, the row
// passes between them and the elementwise updates of rejected attempts) that
// the launch-per-pass sweep (k_col_tan / k_row_tan / k_tan_reject) issues one
// kernel each, for the same batch of tangents at a fixed linearisation
// (reference: jax.jvp of objective_RPO, jax_scripts/lib/utils.py:108, through
// the adaptive stepper of jax_scripts/lib/timestepping.py:151-335).
//
// One thread-block cluster of CL = N / W CTAs of W warps serves one tangent
// (W = 16: 8 CTAs at n = 128, a portable cluster; W = 8: 16 CTAs, half the
// warps per SM and no register cap below 255):
//   * a column pass gives each warp fixed columns (ky, channel) of the box --
//     column c of tangent b on warp c / CL of CTA c % CL -- and runs the same
//     per-column body as k_col_tan (col_tan_body), so the arithmetic and the
//     rounding are those of the launch-per-pass sweep;
//   * a row pass gives CTA r the W physical rows W r .. W r + W - 1, one warp
//     per row, and runs k_row_tan's body (row_tan_body) with W-row tiles;
//   * a rejected attempt updates the tangent's carried k1 column by column on
//     the same warps as the column passes (tan_reject_at).
// Consecutive passes of the same kind (column stages and rejects) touch only
// the warp's own box rows, so they follow each other without a barrier (a
// __syncwarp orders the lanes' writes before the next pass's staged reads).
// Between a column pass and a row pass the cluster synchronises with the
// hardware cluster barrier (arrive.release / wait.acquire), whose
// release/acquire makes one pass's writes visible to the next pass's readers on
// the other SMs of the cluster.  The barrier is a hardware barrier over CTAs
// that are co-scheduled by construction (a cluster), so no wait in this kernel
// spins on memory.
//
// The intermediate arrays between the passes travel one of two ways (template
// flag DSM):
//   * DSM = false: through global memory (G, H; L2-resident at these sizes);
//   * DSM = true: through distributed shared memory -- a column pass writes its
//     inverse transforms straight into the G tiles of the CTAs that own those
//     physical rows (col_uv_to_tiles), and a row pass sends its H tile to the
//     shared rows of the warps that transform those columns (scatter_h_tile),
//     so neither array leaves the cluster.  The first pass of a launch reads and
//     the last one writes global G / H, which carries the state from one launch
//     to the next (a launch ends before a row pass, at a regeneration chunk).
// With DSH (8-warp CTAs only, for shared-memory room) each column warp keeps its
// column's tangent slots ([S_NSLOT][M]) in shared memory for the whole launch:
// loaded at the start, written back to global D at the end.
//
// The same layout runs the primal: k_rk4_chain (fixed-step Lawson-RK4 steps)
// and k_rk43_chain (adaptive attempts with the error norm and the accept/reject
// decision in the kernel), below.
#pragma once

#include "kernels_tan.cuh"

namespace ecs {

enum ChainKind : int { CH_COL = 0, CH_ROW = 1, CH_REJECT = 2 };

// One pass of the sweep.  Record offsets are in box vectors from the record
// base; `item` indexes the physical fields of the launch's regeneration chunk.
struct ChainOp {
  int kind, stage, produce, pad;
  long rec, rec2;
  long item;
  double h;
};

// W warps per CTA = physical rows per CTA in a row pass; CL = N / W CTAs per cluster.
template <int N, int W> __host__ __device__ constexpr int chain_cl() { return N / W; }
// Warps per CTA that own columns in the column passes (2 K columns over CL CTAs).
template <int N, int W> __host__ __device__ constexpr int chain_colwarps() {
  return (2 * ((N - 1) / 3 + 1) + chain_cl<N, W>() - 1) / chain_cl<N, W>();
}
// Operand rows staged per column warp: the largest col_tan_nop over the adaptive
// stages (8), or, with the tangent slots in shared memory (DSH), the largest
// number of record rows a stage reads (5, stage C).
constexpr int CH_NOP = 8, CH_NOP_DSH = 5;
// Shared-memory regions of a chain kernel (offsets in complex entries), with
// `stage` complex entries of column staging per column warp: twiddles; with
// DSM the G tile and the column warps' H rows; the column staging overlaid
// with the row tiles; with DSH the column warps' tangent slots [S_NSLOT][M].
template <int N, int W, bool DSM, bool DSH = false> struct ChainSmem {
  static constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  static constexpr int CW = chain_colwarps<N, W>();
  static constexpr int tw = 0;
  static constexpr int gt = fft_smem(N, W);                        // G tile (DSM)
  static constexpr int hc = gt + (DSM ? NG * K * (W + 1) : 0);     // column warps' H rows (DSM)
  static constexpr int work = hc + (DSM ? CW * 2 * N : 0);         // staging / row tiles
  static constexpr int row = (DSM ? NH : NG + NH) * K * (W + 1);
  static constexpr int ds_at(int stage) { return work + (CW * stage > row ? CW * stage : row); }
  static constexpr int end_at(int stage) { return ds_at(stage) + (DSH ? CW * S_NSLOT * M : 0); }
};
template <typename R, int N, int W, bool DSM, bool DSH = false>
__host__ __device__ constexpr size_t chain_smem_for(int stage) {
  return (size_t)ChainSmem<N, W, DSM, DSH>::end_at(stage) * sizeof(cplx<R>);
}
template <typename R, int N, int W, bool DSM, bool DSH = false> __host__ __device__ constexpr size_t chain_smem() {
  return chain_smem_for<R, N, W, DSM, DSH>((DSH ? CH_NOP_DSH : CH_NOP) * (2 * ((N - 1) / 3) + 1));
}

template <typename R>
struct ChainParams {
  ColTanParams<R> col;   // H, G, D, nslot, dT, t, dscale, tw, nu, eta, B of every column pass
  RowTanParams<R> row;   // G, H, tw of every row pass
  const cplx<R>* rec;    // record base
  const R* phys;         // [item - item0][N][NPH][N]: the regeneration chunk
  long item0;            // first item of the chunk
  const ChainOp* ops;
  int op0, op1;
};

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;\n" ::: "memory");
}

template <typename R, int N, int W, bool DSM, bool DSH>
__device__ __forceinline__ void chain_col(const ChainParams<R>& P, const ChainOp& op, int b, int rank, int w,
                                          int lane, const cplx<R>* s_tw, cplx<R>* my_op, const cplx<R>* hrows,
                                          cplx<R>* gtile, cplx<R>* dsh) {
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  constexpr int CL = chain_cl<N, W>();
  const int c = w * CL + rank;   // this warp's column of the tangent
  if (w >= chain_colwarps<N, W>() || c >= 2 * K) return;
  const int colid = b * 2 * K + c;
  ColTanParams<R> p = P.col;
  p.rec = P.rec + (size_t)op.rec * VEC;
  p.rec2 = P.rec + (size_t)op.rec2 * VEC;
  p.h = op.h;
  p.stage = op.stage;
  p.produce = op.produce;
  if (op.kind == CH_REJECT) {
    const int ch = c & 1, ky = c >> 1;
    cplx<R>* Db = p.D + (size_t)b * p.nslot * VEC;
    const R dpar = (R)(p.dT[b] * p.dscale);
    for (int s = lane; s < M; s += 32) {
      const size_t o = ((size_t)ch * K + ky) * M + s;
      if constexpr (DSH) dsh[S_K1 * M + s] = tan_reject_k1<R>(p.rec, VEC, o, dpar, dsh[S_K1 * M + s]);
      else tan_reject_at<R>(Db, p.rec, VEC, o, dpar);
    }
    return;
  }
  switch (op.stage) {
    case T43_START: col_tan_body<R, N, T43_START, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    case T43_INIT: col_tan_body<R, N, T43_INIT, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    case T43_A: col_tan_body<R, N, T43_A, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    case T43_B: col_tan_body<R, N, T43_B, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    case T43_C: col_tan_body<R, N, T43_C, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    case T43_D: col_tan_body<R, N, T43_D, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    case T43_EA: col_tan_body<R, N, T43_EA, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
    default: col_tan_body<R, N, T43_E, DSM ? W : 0, DSH>(p, colid, lane, s_tw, my_op, hrows, gtile, dsh); break;
  }
}

// Grid: B clusters of CL CTAs (cluster b = tangent b; the cluster shape is a
// launch attribute), W * 32 threads each.
template <typename R, int N, int W, bool DSM, bool DSH>
__global__ void __launch_bounds__(W * 32, 1) k_tan_chain(ChainParams<R> P) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  constexpr int CL = chain_cl<N, W>();
  constexpr int NOPW = DSH ? CH_NOP_DSH : CH_NOP;
  static_assert(N <= 128, "staged column operands need n <= 128");
  static_assert(col_tan_nop<N, T43_C>() <= CH_NOP && col_tan_nop<N, T43_EA>() <= CH_NOP &&
                col_tan_nop<N, T43_A>() <= CH_NOP && col_tan_nop<N, T43_D>() <= CH_NOP, "staging rows");
  static_assert(popc_c(tan_qmask(T43_C)) <= CH_NOP_DSH && popc_c(tan_qmask(T43_EA)) + popc_c(tan_qmask2(T43_EA)) <= CH_NOP_DSH,
                "record rows staged with the slots in shared memory");
  using SM = ChainSmem<N, W, DSM, DSH>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_base = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_tw = s_base + SM::tw;
  cplx<R>* s_gt = s_base + SM::gt;
  cplx<R>* s_hc = s_base + SM::hc;
  cplx<R>* s_work = s_base + SM::work;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x / CL, rank = blockIdx.x - b * CL;
  const int wc = w < chain_colwarps<N, W>() ? w : 0;
  const int cown = w * CL + rank;   // this warp's column (tangent slots in shared memory)
  const bool owns = w < chain_colwarps<N, W>() && cown < 2 * K;
  cplx<R>* dsh = s_base + SM::ds_at(NOPW * M) + (size_t)wc * S_NSLOT * M;
  cplx<R>* dglob = P.col.D + (size_t)b * P.col.nslot * VEC + ((size_t)(cown & 1) * K + (cown >> 1)) * M;
  load_twiddles<R, N>(s_tw, P.col.tw);
  pdl_wait();   // launched with programmatic serialization: the predecessor's writes are visible past here
  if constexpr (DSH) {
    if (owns)
      for (int d = 0; d < S_NSLOT; ++d)
        for (int e = lane; e < M; e += 32) dsh[d * M + e] = dglob[d * VEC + e];
  }
  __syncthreads();
  cplx<R>* my_op = s_work + (size_t)wc * NOPW * M;
  int prev = -1;   // kind class of the previous pass: 0 column-like, 1 row
  for (int i = P.op0; i < P.op1; ++i) {
    const ChainOp op = P.ops[i];
    const int cls = op.kind == CH_ROW ? 1 : 0;
    if (prev >= 0 && (cls != prev || cls == 1)) cluster_barrier();
    else if (prev >= 0) __syncwarp();
    prev = cls;
    const bool first = i == P.op0, last = i == P.op1 - 1;   // global G / H at the launch's ends
    if (cls) {
      RowTanParams<R> rp = P.row;
      rp.phys = P.phys + (size_t)(op.item - P.item0) * N * NPH * N;
      if constexpr (DSM)
        row_tan_body<R, N, W, true>(rp, b, rank * W, s_tw, s_gt, s_work, first, last ? nullptr : s_hc);
      else
        row_tan_body<R, N, W>(rp, b, rank * W, s_tw, s_work, s_work + NG * K * (W + 1));
    } else {
      chain_col<R, N, W, DSM, DSH>(P, op, b, rank, w, lane, s_tw, my_op,
                                   (DSM && !first) ? s_hc + (size_t)wc * 2 * N : nullptr,
                                   (DSM && !last) ? s_gt : nullptr, dsh);
    }
  }
  if constexpr (DSH) {   // the slots back to global memory for the next launch and the JVP output
    __syncwarp();
    if (owns)
      for (int d = 0; d < S_NSLOT; ++d)
        for (int e = lane; e < M; e += 32) dglob[d * VEC + e] = dsh[d * M + e];
  }
  if constexpr (DSM) cluster_barrier();   // no CTA leaves while a peer may still write its shared memory
}

// ---------------------------------------------------------------------------
// Lawson-RK4 steps of the primal (timestepping.lawson_rk4,
// jax_scripts/lib/timestepping.py:69-80) in one launch: cluster b advances
// state b through `steps` steps, each stage a row pass (k_row_rhs's body,
// W-row tiles) and a column pass (k_col_rk4's body), with the same layout and
// barriers as k_tan_chain.  The stage input of the first stage is in G (from a
// COL_START column pass before the launch).
// ---------------------------------------------------------------------------
template <typename R>
struct Rk4ChainParams {
  ColParams<R> col;   // stage and produce are set per stage
  RowParams<R> row;
  long steps;
  int last_produce;   // inverse transforms after the last stage (the next stage input)
};

// per column warp: 3 complex rows (F, A1, K2) and one real row (e), in complex units
template <typename R, int N, int W, bool DSM> __host__ __device__ constexpr size_t rk4_chain_smem() {
  return chain_smem_for<R, N, W, DSM>(4 * (2 * ((N - 1) / 3) + 1));
}

template <typename R, int N, int W, bool DSM>
__global__ void __launch_bounds__(W * 32, 1) k_rk4_chain(Rk4ChainParams<R> P) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int CL = chain_cl<N, W>();
  static_assert(N <= 128, "staged column operands need n <= 128");
  using SM = ChainSmem<N, W, DSM>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_base = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_tw = s_base + SM::tw;
  cplx<R>* s_gt = s_base + SM::gt;
  cplx<R>* s_hc = s_base + SM::hc;
  cplx<R>* s_work = s_base + SM::work;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x / CL, rank = blockIdx.x - b * CL;
  const int cidx = w * CL + rank;   // this warp's column of the state
  const bool has_col = w < chain_colwarps<N, W>() && cidx < 2 * K;
  const int colid = b * 2 * K + cidx;
  cplx<R>* my_c = s_work + (size_t)(has_col ? w : 0) * 4 * M;
  R* my_e = reinterpret_cast<R*>(my_c + 3 * M);
  const cplx<R>* my_h = DSM ? s_hc + (size_t)(has_col ? w : 0) * 2 * N : nullptr;
  load_twiddles<R, N>(s_tw, P.col.tw);
  pdl_wait();   // launched with programmatic serialization: the predecessor's writes are visible past here
  __syncthreads();
  for (long step = 0; step < P.steps; ++step) {
    for (int st = COL_RK4_S1; st <= COL_RK4_S4; ++st) {
      if (step > 0 || st > COL_RK4_S1) cluster_barrier();   // column pass -> row pass
      const bool first = step == 0 && st == COL_RK4_S1, last = step == P.steps - 1 && st == COL_RK4_S4;
      if constexpr (DSM)
        row_rhs_body<R, N, W, true>(P.row, b, rank * W, s_tw, s_gt, s_work, first, s_hc);
      else
        row_rhs_body<R, N, W>(P.row, b, rank * W, s_tw, s_work, s_work + NG * K * (W + 1));
      cluster_barrier();                                     // row pass -> column pass
      if (!has_col) continue;
      ColParams<R> p = P.col;
      p.stage = st;
      p.produce = last ? P.last_produce : 1;
      cplx<R>* gt = (DSM && !last) ? s_gt : nullptr;
      switch (st) {
        case COL_RK4_S1: col_rk4_body<R, N, COL_RK4_S1, DSM ? W : 0>(p, colid, lane, s_tw, my_c, my_e, my_h, gt); break;
        case COL_RK4_S2: col_rk4_body<R, N, COL_RK4_S2, DSM ? W : 0>(p, colid, lane, s_tw, my_c, my_e, my_h, gt); break;
        case COL_RK4_S3: col_rk4_body<R, N, COL_RK4_S3, DSM ? W : 0>(p, colid, lane, s_tw, my_c, my_e, my_h, gt); break;
        default: col_rk4_body<R, N, COL_RK4_S4, DSM ? W : 0>(p, colid, lane, s_tw, my_c, my_e, my_h, gt); break;
      }
    }
  }
  if constexpr (DSM) cluster_barrier();   // no CTA leaves while a peer may still write its shared memory
}

// ---------------------------------------------------------------------------
// Adaptive Lawson-RK4(3) attempts of the primal (timestepping.lawson_rk43,
// jax_scripts/lib/timestepping.py:151-335) in one launch: cluster b runs state
// b's attempts until it completes or `amax` attempts were made -- the column
// stages A..E (k_col_rk43's body), the four RHS row passes (k_row_rhs's body)
// and the error norm (k_row_err's body); each CTA's maximum goes to the
// cluster through distributed shared memory, CTA 0 makes the accept/reject
// decision and the step-size update on the control block (rk43_control, as
// the last block of k_row_err does), and every CTA reads it after the next
// cluster barrier.  The G and H arrays go through global memory.  Set-up,
// START and INIT passes run before the launch.
// ---------------------------------------------------------------------------
template <typename R>
struct Rk43ChainParams {
  Col43Params<R> col;
  RowParams<R> row;
  double atol;
  double* rec_h;   // optional [B][cap] attempted step sizes
  int* rec_acc;    // optional [B][cap] accept flags
  long amax;       // attempts at most
};
constexpr int CH_NOP43 = 5;   // rows staged per column warp by an attempt stage (slots + forcing)

template <typename R, int N, int W> __host__ __device__ constexpr size_t rk43_chain_smem() {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr size_t col = (size_t)chain_colwarps<N, W>() * CH_NOP43 * M;
  constexpr size_t row = (size_t)(NG + NH) * K * (W + 1);
  return (fft_smem(N, W) + (col > row ? col : row)) * sizeof(cplx<R>);
}

template <typename R, int N, int W>
__global__ void __launch_bounds__(W * 32, 1) k_rk43_chain(Rk43ChainParams<R> P) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int CL = chain_cl<N, W>();
  static_assert(N <= 128, "staged column operands need n <= 128");
  static_assert(col_rk43_nop<N, R43_C>() <= CH_NOP43 && col_rk43_nop<N, R43_D>() <= CH_NOP43 &&
                col_rk43_nop<N, R43_B>() <= CH_NOP43 && col_rk43_nop<N, R43_E>() <= CH_NOP43, "staging rows");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_work = s_tw + fft_smem(N, W);
  __shared__ double s_max[W];
  __shared__ double s_part;   // this CTA's error maximum, read by CTA 0 of the cluster
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x / CL, rank = blockIdx.x - b * CL;
  const int cidx = w * CL + rank;   // this warp's column of the state
  const bool has_col = w < chain_colwarps<N, W>() && cidx < 2 * K;
  const int colid = b * 2 * K + cidx;
  cplx<R>* my_op = s_work + (size_t)(has_col ? w : 0) * CH_NOP43 * M;
  StepCtl* ctl = P.col.ctl + b;
  load_twiddles<R, N>(s_tw, P.col.tw);
  pdl_wait();   // launched with programmatic serialization: the predecessor's writes are visible past here
  __syncthreads();
  for (long a = 0; a < P.amax; ++a) {
    if (*(volatile int*)&ctl->done) break;   // written by CTA 0 before the last cluster barrier
    if (has_col) col_rk43_body<R, N, R43_A>(P.col, colid, lane, s_tw, my_op);
    cluster_barrier();
#pragma unroll 1
    for (int st = R43_B; st <= R43_E; ++st) {
      row_rhs_body<R, N, W>(P.row, b, rank * W, s_tw, s_work, s_work + NG * K * (W + 1));
      cluster_barrier();
      if (has_col) {
        switch (st) {
          case R43_B: col_rk43_body<R, N, R43_B>(P.col, colid, lane, s_tw, my_op); break;
          case R43_C: col_rk43_body<R, N, R43_C>(P.col, colid, lane, s_tw, my_op); break;
          case R43_D: col_rk43_body<R, N, R43_D>(P.col, colid, lane, s_tw, my_op); break;
          default: col_rk43_body<R, N, R43_E>(P.col, colid, lane, s_tw, my_op); break;
        }
      }
      cluster_barrier();
    }
    const double bm = row_err_max<R, N, W>(P.col.G, b, rank * W, s_tw, s_work, s_max);
    if (threadIdx.x == 0) s_part = bm;
    cluster_barrier();
    if (rank == 0 && threadIdx.x == 0) {
      cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
      double err = 0.0;
      for (int r = 0; r < CL; ++r) {
        const double q = *cl.map_shared_rank(&s_part, (unsigned)r);
        err = (q > err || isnan(q)) ? q : err;
      }
      const int at = ctl->attempts, cap = P.col.cap;
      rk43_control(*ctl, P.atol, err, P.rec_h && at < cap ? P.rec_h + (size_t)b * cap : nullptr,
                   P.rec_acc && at < cap ? P.rec_acc + (size_t)b * cap : nullptr);
    }
    cluster_barrier();
  }
}

}  // namespace ecs
