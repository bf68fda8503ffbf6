// Cluster-resident tangent sweep of the adaptive Lawson-RK4(3) linearisation:
// one launch runs a whole list of tangent passes (the column stages, the row
// passes between them and the elementwise updates of rejected attempts) that
// the launch-per-pass sweep (k_col_tan / k_row_tan / k_tan_reject) issues one
// kernel each, for the same batch of tangents at a fixed linearisation
// (reference: jax.jvp of objective_RPO, jax_scripts/lib/utils.py:108, through
// the adaptive stepper of jax_scripts/lib/timestepping.py:151-335).
//
// One thread-block cluster of CL = N / 16 CTAs of 16 warps serves one tangent:
//   * a column pass gives each warp fixed columns (ky, channel) of the box --
//     column c of tangent b on warp c / CL of CTA c % CL -- and runs the same
//     per-column body as k_col_tan (col_tan_body), so the arithmetic and the
//     rounding are those of the launch-per-pass sweep;
//   * a row pass gives CTA r the 16 physical rows 16 r .. 16 r + 15, one warp
//     per row, and runs k_row_tan's body (row_tan_body) with 16-row tiles;
//   * a rejected attempt updates the tangent's carried k1 column by column on
//     the same warps as the column passes (tan_reject_at).
// Consecutive passes of the same kind (column stages and rejects) touch only
// the warp's own box rows, so they follow each other without a barrier (a
// __syncwarp orders the lanes' writes before the next pass's staged reads).
// Between a column pass and a row pass the cluster synchronises with the
// hardware cluster barrier (arrive.release / wait.acquire): the G and H
// intermediate arrays stay in global memory (L2-resident at these sizes), and
// the barrier's release/acquire makes one pass's writes visible to the next
// pass's readers on the other SMs of the cluster.  The barrier is a hardware
// barrier over CTAs that are co-scheduled by construction (a cluster), so no
// wait in this kernel spins on memory.
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

constexpr int CH_WARPS = 16;   // warps per CTA = physical rows per CTA in a row pass
template <int N> __host__ __device__ constexpr int chain_cl() { return N / CH_WARPS; }
// Warps per CTA that own columns in the column passes (2 K columns over CL CTAs).
template <int N> __host__ __device__ constexpr int chain_colwarps() {
  return (2 * ((N - 1) / 3 + 1) + chain_cl<N>() - 1) / chain_cl<N>();
}
// Operand rows staged per column warp: the largest col_tan_nop over the adaptive stages.
constexpr int CH_NOP = 8;
template <typename R, int N> __host__ __device__ constexpr size_t chain_smem() {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr size_t col = (size_t)chain_colwarps<N>() * CH_NOP * M;
  constexpr size_t row = (size_t)(NG + NH) * K * (CH_WARPS + 1);
  return (fft_smem(N, CH_WARPS) + (col > row ? col : row)) * sizeof(cplx<R>);
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

template <typename R, int N>
__device__ __forceinline__ void chain_col(const ChainParams<R>& P, const ChainOp& op, int b, int rank, int w,
                                          int lane, const cplx<R>* s_tw, cplx<R>* my_op) {
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  constexpr int CL = chain_cl<N>();
  const int c = w * CL + rank;   // this warp's column of the tangent
  if (w >= chain_colwarps<N>() || c >= 2 * K) return;
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
    for (int s = lane; s < M; s += 32) tan_reject_at<R>(Db, p.rec, VEC, ((size_t)ch * K + ky) * M + s, dpar);
    return;
  }
  switch (op.stage) {
    case T43_START: col_tan_body<R, N, T43_START>(p, colid, lane, s_tw, my_op); break;
    case T43_INIT: col_tan_body<R, N, T43_INIT>(p, colid, lane, s_tw, my_op); break;
    case T43_A: col_tan_body<R, N, T43_A>(p, colid, lane, s_tw, my_op); break;
    case T43_B: col_tan_body<R, N, T43_B>(p, colid, lane, s_tw, my_op); break;
    case T43_C: col_tan_body<R, N, T43_C>(p, colid, lane, s_tw, my_op); break;
    case T43_D: col_tan_body<R, N, T43_D>(p, colid, lane, s_tw, my_op); break;
    case T43_EA: col_tan_body<R, N, T43_EA>(p, colid, lane, s_tw, my_op); break;
    default: col_tan_body<R, N, T43_E>(p, colid, lane, s_tw, my_op); break;
  }
}

// Grid: B clusters of CL CTAs (cluster b = tangent b), CH_WARPS * 32 threads each.
template <typename R, int N>
__global__ void __cluster_dims__(chain_cl<N>(), 1, 1) __launch_bounds__(CH_WARPS * 32, 1)
k_tan_chain(ChainParams<R> P) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int CL = chain_cl<N>();
  static_assert(N <= 128, "staged column operands need n <= 128");
  static_assert(col_tan_nop<N, T43_C>() <= CH_NOP && col_tan_nop<N, T43_EA>() <= CH_NOP &&
                col_tan_nop<N, T43_A>() <= CH_NOP && col_tan_nop<N, T43_D>() <= CH_NOP, "staging rows");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_work = s_tw + fft_smem(N, CH_WARPS);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x / CL, rank = blockIdx.x - b * CL;
  load_twiddles<R, N>(s_tw, P.col.tw);
  pdl_wait();   // launched with programmatic serialization: the predecessor's writes are visible past here
  __syncthreads();
  cplx<R>* my_op = s_work + (size_t)(w < chain_colwarps<N>() ? w : 0) * CH_NOP * M;
  int prev = -1;   // kind class of the previous pass: 0 column-like, 1 row
  for (int i = P.op0; i < P.op1; ++i) {
    const ChainOp op = P.ops[i];
    const int cls = op.kind == CH_ROW ? 1 : 0;
    if (prev >= 0 && (cls != prev || cls == 1)) cluster_barrier();
    else if (prev >= 0) __syncwarp();
    prev = cls;
    if (cls) {
      RowTanParams<R> rp = P.row;
      rp.phys = P.phys + (size_t)(op.item - P.item0) * N * NPH * N;
      row_tan_body<R, N, CH_WARPS>(rp, b, rank * CH_WARPS, s_tw, s_work, s_work + NG * K * (CH_WARPS + 1));
    } else {
      chain_col<R, N>(P, op, b, rank, w, lane, s_tw, my_op);
    }
  }
}

// ---------------------------------------------------------------------------
// Lawson-RK4 steps of the primal (timestepping.lawson_rk4,
// jax_scripts/lib/timestepping.py:69-80) in one launch: cluster b advances
// state b through `steps` steps, each stage a row pass (k_row_rhs's body,
// 16-row tiles) and a column pass (k_col_rk4's body), with the same layout and
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

template <typename R, int N> __host__ __device__ constexpr size_t rk4_chain_smem() {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  // per column warp: 3 complex rows (F, A1, K2) and one real row (e), in complex units
  constexpr size_t col = (size_t)chain_colwarps<N>() * 4 * M;
  constexpr size_t row = (size_t)(NG + NH) * K * (CH_WARPS + 1);
  return (fft_smem(N, CH_WARPS) + (col > row ? col : row)) * sizeof(cplx<R>);
}

template <typename R, int N>
__global__ void __cluster_dims__(chain_cl<N>(), 1, 1) __launch_bounds__(CH_WARPS * 32, 1)
k_rk4_chain(Rk4ChainParams<R> P) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int CL = chain_cl<N>();
  static_assert(N <= 128, "staged column operands need n <= 128");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_work = s_tw + fft_smem(N, CH_WARPS);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b = blockIdx.x / CL, rank = blockIdx.x - b * CL;
  const int cidx = w * CL + rank;   // this warp's column of the state
  const bool has_col = w < chain_colwarps<N>() && cidx < 2 * K;
  const int colid = b * 2 * K + cidx;
  cplx<R>* my_c = s_work + (size_t)(has_col ? w : 0) * 4 * M;
  R* my_e = reinterpret_cast<R*>(my_c + 3 * M);
  load_twiddles<R, N>(s_tw, P.col.tw);
  pdl_wait();   // launched with programmatic serialization: the predecessor's writes are visible past here
  __syncthreads();
  for (long step = 0; step < P.steps; ++step) {
    for (int st = COL_RK4_S1; st <= COL_RK4_S4; ++st) {
      if (step > 0 || st > COL_RK4_S1) cluster_barrier();   // column pass -> row pass
      row_rhs_body<R, N, CH_WARPS>(P.row, b, rank * CH_WARPS, s_tw, s_work, s_work + NG * K * (CH_WARPS + 1));
      cluster_barrier();                                     // row pass -> column pass
      if (!has_col) continue;
      ColParams<R> p = P.col;
      p.stage = st;
      p.produce = (st == COL_RK4_S4 && step == P.steps - 1) ? P.last_produce : 1;
      switch (st) {
        case COL_RK4_S1: col_rk4_body<R, N, COL_RK4_S1>(p, colid, lane, s_tw, my_c, my_e); break;
        case COL_RK4_S2: col_rk4_body<R, N, COL_RK4_S2>(p, colid, lane, s_tw, my_c, my_e); break;
        case COL_RK4_S3: col_rk4_body<R, N, COL_RK4_S3>(p, colid, lane, s_tw, my_c, my_e); break;
        default: col_rk4_body<R, N, COL_RK4_S4>(p, colid, lane, s_tw, my_c, my_e); break;
      }
    }
  }
}

}  // namespace ecs
