// Templated host orchestration of the kernels for one (dtype, n): launch
// helpers, the Impl<R, N> operations and the context initialisation.
// Included by one instantiation unit per (dtype, n) (inst_*.cu).
#pragma once

#include "../../include/ecs_mhd.h"
#include "kernels.cuh"
#include "kernels_rk43.cuh"
#include "kernels_tan.cuh"
#include "kernels_adj.cuh"
#include "kernels_fx.cuh"
#include "kernels_fxl.cuh"
#include "kernels_chain.cuh"
#include "api_internal.cuh"
#include "impl_table.h"

#include <algorithm>
#include <numeric>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <utility>
#include <type_traits>
#include <mutex>

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
namespace ecs {

constexpr int XT = 8;
constexpr int COLWARPS = 4;

// Row kernels with NG (or 3 adjoint) input and NH (or NHA adjoint) output tiles: 7 tiles of K x (X+1).
template <typename R, int N, int X = XT> size_t smem_row_rhs() { return (fft_smem(N, X) + 7 * Geomc<N>::K * (X + 1)) * sizeof(cplx<R>); }
// Small batches use 2-row tiles: 4x more CTAs for the same rows.
constexpr int XTS = 2;
template <int N> bool small_rows(int B) { return (long)B * (N / XT) < 2L * 148; }
template <typename R, int N> size_t smem_row_tan2() { return (fft_smem(N, XT) + 11 * Geomc<N>::K * (XT + 1)) * sizeof(cplx<R>); }
template <typename R, int N> size_t smem_row_phys() { return (fft_smem(N, XT) + NG * Geomc<N>::K * (XT + 1)) * sizeof(cplx<R>); }
template <typename R, int N, int X = XT> size_t smem_row_2f() { return (fft_smem(N, X) + 2 * Geomc<N>::K * (X + 1)) * sizeof(cplx<R>); }

// Launch a stepping kernel of batch B; with c->pdl set, with programmatic
// stream serialization (the kernel waits on its predecessor itself, see
// pdl_wait), so that a kernel's launch and prologue overlap its predecessor's
// tail.  Measured at n=128 FP64: the batch-64 tangent kernels gain 5-7%, and
// single-state chains inside CUDA graphs gain 10-24% (gradient, plain JVP,
// Lawson-RK4), except the pipelined linearisation's primal (see below).
template <typename... P, typename... A>
inline void launch_step(ecs_ctx* c, int B, void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                        A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  // inside a PlainOrder scope small batches keep plain stream order (see PlainOrder)
  const bool plain = c->plain_order > 0 && B < 8;
  cfg.attrs = at; cfg.numAttrs = (c->pdl && B >= c->pdl_minb && !plain) ? 1 : 0;
  ++c->launches;
  cudaLaunchKernelEx(&cfg, k, args...);
}

// launch_step for a kernel launched as clusters of `cl` CTAs along x.
template <typename... P, typename... A>
inline void launch_cluster(ecs_ctx* c, int B, int cl, void (*k)(P...), dim3 grid, dim3 block, size_t smem,
                           cudaStream_t s, A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid; cfg.blockDim = block; cfg.dynamicSmemBytes = smem; cfg.stream = s;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cl; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = 1;
  const bool plain = c->plain_order > 0 && B < 8;
  cfg.attrs = at; cfg.numAttrs = (c->pdl && B >= c->pdl_minb && !plain) ? 2 : 1;
  ++c->launches;
  cudaLaunchKernelEx(&cfg, k, args...);
}

// Scope in which batches below 8 launch without programmatic dependent launch:
// the adaptive Lawson-RK4(3) solve and the fixed-step integrations measured
// 5-10% slower with it at batch 1, and the batch-1 primal that runs beside the
// tangent batch (pipelined linearisation) would park early-launched CTAs on
// SMs that the tangents need.  Graphs captured inside the scope keep it.
struct PlainOrder {
  ecs_ctx* c;
  explicit PlainOrder(ecs_ctx* c_) : c(c_) { ++c->plain_order; }
  ~PlainOrder() { --c->plain_order; }
  PlainOrder(const PlainOrder&) = delete;
  PlainOrder& operator=(const PlainOrder&) = delete;
};

template <typename R, int N, int W>
int configure_chain() {
  int st = 0;
  auto attrs = [&](auto* k, size_t smem) {
    st |= (int)cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (chain_cl<N, W>() > 8) st |= (int)cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  };
  attrs(k_tan_chain<R, N, W, false, false>, chain_smem<R, N, W, false, false>());
  attrs(k_tan_chain<R, N, W, true, false>, chain_smem<R, N, W, true, false>());
  if constexpr (W == 8) {   // tangent slots in shared memory: the 8-warp shape only (smem)
    attrs(k_tan_chain<R, N, W, false, true>, chain_smem<R, N, W, false, true>());
    attrs(k_tan_chain<R, N, W, true, true>, chain_smem<R, N, W, true, true>());
  }
  attrs(k_rk43_chain<R, N, W>, rk43_chain_smem<R, N, W>());
  attrs(k_rk4_chain<R, N, W, false>, rk4_chain_smem<R, N, W, false>());
  attrs(k_rk4_chain<R, N, W, true>, rk4_chain_smem<R, N, W, true>());
  return st;
}

// Clusters of the W-warp tangent chain kernel (its variant with the largest
// shared memory) that the device holds at once; 0 if it cannot hold one.
template <typename R, int N, int W>
int chain_clusters() {
  constexpr bool DSH = W == 8;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(chain_cl<N, W>()); cfg.blockDim = dim3(W * 32); cfg.dynamicSmemBytes = chain_smem<R, N, W, true, DSH>();
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)chain_cl<N, W>(); at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  cfg.attrs = at; cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, k_tan_chain<R, N, W, true, DSH>, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

template <typename R, int N>
int configure_kernels(ecs_ctx* c) {
  int st = ECS_OK;
  st |= (int)cudaFuncSetAttribute(k_row_rhs<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_to_box<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_from_box<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_err<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_phys<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_phys<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_tan<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_adj<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_tan2<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_tan2<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_adj2<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_rhs<R, N, XTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N, XTS>());
  st |= (int)cudaFuncSetAttribute(k_row_err<R, N, XTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N, XTS>());
  st |= (int)cudaFuncSetAttribute(k_row_tan<R, N, XTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N, XTS>());
  st |= (int)cudaFuncSetAttribute(k_row_tan<R, N, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N, 4>());
  st |= (int)cudaFuncSetAttribute(k_row_adj<R, N, XTS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N, XTS>());
  if constexpr (N <= 128) {
    st |= configure_chain<R, N, 8>();
    st |= configure_chain<R, N, 16>();
  }
  if (st) return cuda_err(c, cudaGetLastError(), "cudaFuncSetAttribute");
  if constexpr (N <= 128) {
    // clusters of each chain shape that the device holds at once (8 warps:
    // clusters of N / 8 CTAs, non-portable above 8; 16 warps: N / 16 CTAs)
    c->chain_res8 = chain_clusters<R, N, 8>();
    c->chain_res16 = chain_clusters<R, N, 16>();
  }
  return ECS_OK;
}



template <typename R, int N>
void launch_row_to_box(ecs_ctx* c, const R* fields, cplx<R>* H, int B, cudaStream_t s) {
  RowFwdParams<R> p; p.fields = fields; p.H = H; p.tw = (const cplx<R>*)c->tw; p.B = B;
  ++c->launches; k_row_to_box<R, N, XT><<<B * (N / XT), XT * 32, smem_row_2f<R, N>(), s>>>(p);
}

template <typename R, int N>
void launch_col_to_box(ecs_ctx* c, const cplx<R>* H, cplx<R>* V, int B, int nf, cudaStream_t s, long vstride = 0) {
  ColBoxParams<R> p; p.H = H; p.V = V; p.tw = (const cplx<R>*)c->tw; p.B = B; p.nf = nf;
  p.vstride = vstride > 0 ? vstride : (long)nf * Geomc<N>::K * Geomc<N>::M;
  const int cols = B * nf * Geomc<N>::K;
  ++c->launches; k_col_to_box<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
}

template <typename R, int N>
void launch_col_from_box(ecs_ctx* c, const cplx<R>* V, cplx<R>* G2, int B, const double* sx, int ny, int rot,
                         int use_sym, int mult_ikx, cudaStream_t s, int sx_shared = 0) {
  ColFromBoxParams<R> p; p.V = V; p.G = G2; p.tw = (const cplx<R>*)c->tw; p.sx = sx; p.sx_shared = sx_shared;
  p.sy = (ny * 2 * M_PI) / 8;   // symmetry.py:11 s = (n*2*pi)/8
  p.odd = (ny % 2 + 2) % 2 == 1; p.rot = rot; p.use_sym = use_sym; p.mult_ikx = mult_ikx; p.B = B;
  const int cols = B * 2 * Geomc<N>::K;
  ++c->launches; k_col_from_box<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
}

template <typename R, int N>
void launch_row_from_box(ecs_ctx* c, const cplx<R>* G2, R* out, const R* base, double* rowsq, int B, int mode,
                         cudaStream_t s) {
  RowFromBoxParams<R> p; p.G = G2; p.out = out; p.base = base; p.rowsq = rowsq; p.tw = (const cplx<R>*)c->tw;
  p.B = B; p.mode = mode;
  ++c->launches; k_row_from_box<R, N, XT><<<B * (N / XT), XT * 32, smem_row_2f<R, N>(), s>>>(p);
}

template <typename R, int N>
void launch_col_rk4(ecs_ctx* c, int B, int stage, int produce, int diss, cudaStream_t s, cplx<R>* rec = nullptr,
                    long rec_bstride = 0, int use_done = 0) {
  ColParams<R> p{};
  p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.F = (cplx<R>*)c->F; p.A1 = (cplx<R>*)c->A1;
  p.K2 = (cplx<R>*)c->K2; p.OUT = (cplx<R>*)c->OUT; p.Etab = (const R*)c->Etab; p.ctl = c->ctl;
  p.fhat = (const cplx<R>*)c->fhat; p.tw = (const cplx<R>*)c->tw; p.nu = (R)c->nu; p.eta = (R)c->eta;
  p.B = B; p.stage = stage; p.produce = produce; p.diss = diss; p.rec = rec; p.rec_bstride = rec_bstride;
  p.use_done = use_done;
  const int cols = B * Geomc<N>::K * 2;   // one warp per (batch, ky, channel)
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  switch (stage) {
    case COL_START: launch_step(c, B, k_col_rk4<R, N, COL_START>, g, bl, 0, s, p); break;
    case COL_RK4_S1: launch_step(c, B, k_col_rk4<R, N, COL_RK4_S1>, g, bl, 0, s, p); break;
    case COL_RK4_S2: launch_step(c, B, k_col_rk4<R, N, COL_RK4_S2>, g, bl, 0, s, p); break;
    case COL_RK4_S3: launch_step(c, B, k_col_rk4<R, N, COL_RK4_S3>, g, bl, 0, s, p); break;
    case COL_RK4_S4: launch_step(c, B, k_col_rk4<R, N, COL_RK4_S4>, g, bl, 0, s, p); break;
    default: launch_step(c, B, k_col_rk4<R, N, COL_PLAIN>, g, bl, 0, s, p); break;
  }
}

template <typename R, int N>
void launch_row_rhs(ecs_ctx* c, int B, cudaStream_t s, const StepCtl* ctl = nullptr, R* phys = nullptr,
                    long phys_bstride = 0) {
  RowParams<R> p{}; p.G = (const cplx<R>*)c->G; p.H = (cplx<R>*)c->H; p.tw = (const cplx<R>*)c->tw; p.ctl = ctl;
  p.phys = phys; p.phys_bstride = phys_bstride;
  p.b0x = (R)c->b0x; p.b0y = (R)c->b0y; p.B = B;
  if (small_rows<N>(B)) launch_step(c, B, k_row_rhs<R, N, XTS>, dim3(B * (N / XTS)), dim3(XTS * 32), smem_row_rhs<R, N, XTS>(), s, p);
  else launch_step(c, B, k_row_rhs<R, N, XT>, dim3(B * (N / XT)), dim3(XT * 32), smem_row_rhs<R, N>(), s, p);
}

template <typename R, int N>
void launch_col_rk43(ecs_ctx* c, int B, int stage, cudaStream_t s, cplx<R>* rec = nullptr, int cap = 0) {
  Col43Params<R> p{};
  p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.S = (cplx<R>*)c->S43; p.ctl = c->ctl;
  p.fhat = (const cplx<R>*)c->fhat; p.tw = (const cplx<R>*)c->tw; p.rec = rec; p.cap = cap;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B; p.stage = stage;
  const int cols = B * Geomc<N>::K * 2;   // one warp per (batch, ky, channel)
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  switch (stage) {
    case R43_START: launch_step(c, B, k_col_rk43<R, N, R43_START>, g, bl, 0, s, p); break;
    case R43_INIT: launch_step(c, B, k_col_rk43<R, N, R43_INIT>, g, bl, 0, s, p); break;
    case R43_A: launch_step(c, B, k_col_rk43<R, N, R43_A>, g, bl, 0, s, p); break;
    case R43_B: launch_step(c, B, k_col_rk43<R, N, R43_B>, g, bl, 0, s, p); break;
    case R43_C: launch_step(c, B, k_col_rk43<R, N, R43_C>, g, bl, 0, s, p); break;
    case R43_D: launch_step(c, B, k_col_rk43<R, N, R43_D>, g, bl, 0, s, p); break;
    default: launch_step(c, B, k_col_rk43<R, N, R43_E>, g, bl, 0, s, p); break;
  }
}

template <typename R, int N>
void launch_row_err(ecs_ctx* c, int B, double atol, cudaStream_t s, double* rec_h = nullptr, int* rec_acc = nullptr,
                    int cap = 0) {
  RowErrParams<R> p; p.G = (const cplx<R>*)c->G; p.ctl = c->ctl; p.tw = (const cplx<R>*)c->tw; p.atol = atol;
  p.rec_h = rec_h; p.rec_acc = rec_acc; p.cap = cap; p.B = B;
  if (small_rows<N>(B)) launch_step(c, B, k_row_err<R, N, XTS>, dim3(B * (N / XTS)), dim3(XTS * 32), smem_row_2f<R, N, XTS>(), s, p);
  else launch_step(c, B, k_row_err<R, N, XT>, dim3(B * (N / XT)), dim3(XT * 32), smem_row_2f<R, N>(), s, p);
}

template <typename R, int N>
void launch_regen(ecs_ctx* c, const cplx<R>* rec, const long* items, int nitems, cudaStream_t s, R* phys = nullptr,
                  bool mean = true) {
  ColRegenParams<R> p; p.rec = rec; p.items = items; p.G = (cplx<R>*)c->Greg; p.tw = (const cplx<R>*)c->tw;
  p.nitems = nitems;
  const int cols = nitems * Geomc<N>::K * 2;
  ++c->launches; k_col_regen<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
  RowPhysParams<R> q; q.G = (const cplx<R>*)c->Greg; q.phys = phys ? phys : (R*)c->Phys; q.tw = (const cplx<R>*)c->tw;
  q.b0x = mean ? (R)c->b0x : R(0); q.b0y = mean ? (R)c->b0y : R(0); q.nitems = nitems;   // no mean field in derivatives
  ++c->launches; k_row_phys<R, N, XT><<<nitems * (N / XT), XT * 32, smem_row_phys<R, N>(), s>>>(q);
}

template <typename R, int N>
void launch_row_tan(ecs_ctx* c, int B, const R* phys, cudaStream_t s, long phys_bstride = 0,
                    const StepCtl* ctl = nullptr) {
  RowTanParams<R> p{}; p.ctl = ctl; p.G = (const cplx<R>*)c->G; p.H = (cplx<R>*)c->H; p.phys = phys; p.tw = (const cplx<R>*)c->tw;
  p.B = B; p.phys_bstride = phys_bstride;
  if (small_rows<N>(B)) launch_step(c, B, k_row_tan<R, N, XTS>, dim3(B * (N / XTS)), dim3(XTS * 32), smem_row_rhs<R, N, XTS>(), s, p);
  else if (N == 128 && c->rowtan_xt == 4)   // 4-row tiles measured faster at n = 128 only
    launch_step(c, B, k_row_tan<R, N, 4>, dim3(B * (N / 4)), dim3(4 * 32), smem_row_rhs<R, N, 4>(), s, p);
  else launch_step(c, B, k_row_tan<R, N, XT>, dim3(B * (N / XT)), dim3(XT * 32), smem_row_rhs<R, N>(), s, p);
}

template <typename R, int N>
void launch_col_tan(ecs_ctx* c, int B, int stage, int produce, const cplx<R>* rec, const double* dT, double t,
                    double h, double dscale, int nslot, cudaStream_t s, const StepCtl* ctl = nullptr,
                    long rec_bstride = 0, const double* dscale_b = nullptr, const R* etab = nullptr,
                    const cplx<R>* rec2 = nullptr) {
  ColTanParams<R> p{}; p.ctl = ctl; p.rec_bstride = rec_bstride; p.dscale_b = dscale_b; p.etab = etab;
  p.rec2 = rec2; p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.D = (cplx<R>*)c->D; p.nslot = nslot;
  p.rec = rec; p.dT = dT; p.t = t; p.h = h; p.dscale = dscale; p.tw = (const cplx<R>*)c->tw;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B; p.stage = stage; p.produce = produce;
  const int cols = B * Geomc<N>::K * 2;   // one warp per (batch, ky, channel)
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  switch (stage) {
    case TS_START: launch_step(c, B, k_col_tan<R, N, TS_START>, g, bl, 0, s, p); break;
    case T4_S1: launch_step(c, B, k_col_tan<R, N, T4_S1>, g, bl, 0, s, p); break;
    case T4_S2: launch_step(c, B, k_col_tan<R, N, T4_S2>, g, bl, 0, s, p); break;
    case T4_S3: launch_step(c, B, k_col_tan<R, N, T4_S3>, g, bl, 0, s, p); break;
    case T4_S4: launch_step(c, B, k_col_tan<R, N, T4_S4>, g, bl, 0, s, p); break;
    case T43_START: launch_step(c, B, k_col_tan<R, N, T43_START>, g, bl, 0, s, p); break;
    case T43_INIT: launch_step(c, B, k_col_tan<R, N, T43_INIT>, g, bl, 0, s, p); break;
    case T43_A: launch_step(c, B, k_col_tan<R, N, T43_A>, g, bl, 0, s, p); break;
    case T43_B: launch_step(c, B, k_col_tan<R, N, T43_B>, g, bl, 0, s, p); break;
    case T43_C: launch_step(c, B, k_col_tan<R, N, T43_C>, g, bl, 0, s, p); break;
    case T43_D: launch_step(c, B, k_col_tan<R, N, T43_D>, g, bl, 0, s, p); break;
    case T43_EA: launch_step(c, B, k_col_tan<R, N, T43_EA>, g, bl, 0, s, p); break;
    default: launch_step(c, B, k_col_tan<R, N, T43_E>, g, bl, 0, s, p); break;
  }
}

template <typename R, int N>
void launch_row_adj(ecs_ctx* c, int B, const R* phys, cudaStream_t s, long phys_bstride = 0,
                    const StepCtl* ctl = nullptr) {
  RowAdjParams<R> p{}; p.G = (const cplx<R>*)c->G; p.H = (cplx<R>*)c->H; p.phys = phys; p.tw = (const cplx<R>*)c->tw;
  p.phys_bstride = phys_bstride; p.ctl = ctl;
  p.B = B;
  if (small_rows<N>(B)) launch_step(c, B, k_row_adj<R, N, XTS>, dim3(B * (N / XTS)), dim3(XTS * 32), smem_row_rhs<R, N, XTS>(), s, p);
  else launch_step(c, B, k_row_adj<R, N, XT>, dim3(B * (N / XT)), dim3(XT * 32), smem_row_rhs<R, N>(), s, p);
}

template <typename R, int N>
void launch_col_adj(ecs_ctx* c, int B, int stage, const cplx<R>* rec, const cplx<R>* rec_prev, double t, double h,
                    int nslot, cudaStream_t s, const StepCtl* ctl = nullptr, long rec_bstride = 0) {
  ColAdjParams<R> p{}; p.ctl = ctl; p.rec_bstride = rec_bstride; p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.J = (cplx<R>*)c->D; p.nslot = nslot;
  p.rec = rec; p.rec_prev = rec_prev; p.hacc = c->hacc; p.t = t; p.h = h; p.tw = (const cplx<R>*)c->tw;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B; p.stage = stage;
  const int cols = B * Geomc<N>::K * 2;   // one warp per (batch, ky, channel)
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  switch (stage) {
    case AJ_PRE: launch_step(c, B, k_col_adj<R, N, AJ_PRE>, g, bl, 0, s, p); break;
    case AJ_S4: launch_step(c, B, k_col_adj<R, N, AJ_S4>, g, bl, 0, s, p); break;
    case AJ_S3: launch_step(c, B, k_col_adj<R, N, AJ_S3>, g, bl, 0, s, p); break;
    case AJ_S2: launch_step(c, B, k_col_adj<R, N, AJ_S2>, g, bl, 0, s, p); break;
    case AJ_S1: launch_step(c, B, k_col_adj<R, N, AJ_S1>, g, bl, 0, s, p); break;
    case AJ43_INIT: launch_step(c, B, k_col_adj<R, N, AJ43_INIT>, g, bl, 0, s, p); break;
    case AJ43_PRE: launch_step(c, B, k_col_adj<R, N, AJ43_PRE>, g, bl, 0, s, p); break;
    case AJ43_S5: launch_step(c, B, k_col_adj<R, N, AJ43_S5>, g, bl, 0, s, p); break;
    case AJ43_S4: launch_step(c, B, k_col_adj<R, N, AJ43_S4>, g, bl, 0, s, p); break;
    case AJ43_S3: launch_step(c, B, k_col_adj<R, N, AJ43_S3>, g, bl, 0, s, p); break;
    case AJ43_S2: launch_step(c, B, k_col_adj<R, N, AJ43_S2>, g, bl, 0, s, p); break;
    default: launch_step(c, B, k_col_adj<R, N, AJ43_IPRE>, g, bl, 0, s, p); break;
  }
}

template <typename R, int N, int SCHEME, int... ST>
void launch_col_fx_sw(ecs_ctx* c, int B, int stage, cudaStream_t s, const ColFxParams<R>& p,
                      std::integer_sequence<int, ST...>) {
  const int cols = B * Geomc<N>::K * 2;   // one warp per (batch, ky, channel)
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  ((stage == ST ? launch_step(c, B, k_col_fx<R, N, SCHEME, ST>, g, bl, 0, s, p) : void()), ...);
}

template <typename R, int N>
void launch_col_fx(ecs_ctx* c, int B, int scheme, int stage, int produce, cudaStream_t s, cplx<R>* rec = nullptr) {
  ColFxParams<R> p;
  p.rec = rec;
  p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.S = (cplx<R>*)c->S43; p.Etab = (const R*)c->Etab; p.ctl = c->ctl;
  p.fhat = (const cplx<R>*)c->fhat; p.tw = (const cplx<R>*)c->tw; p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B;
  p.produce = produce;
  if (scheme == FX_RK4) launch_col_fx_sw<R, N, FX_RK4>(c, B, stage, s, p, std::make_integer_sequence<int, 5>{});
  else if (scheme == FX_RK6) launch_col_fx_sw<R, N, FX_RK6>(c, B, stage, s, p, std::make_integer_sequence<int, 9>{});
  else launch_col_fx_sw<R, N, FX_TD4>(c, B, stage, s, p, std::make_integer_sequence<int, 5>{});
}

template <typename R, int N>
void launch_row_tan2(ecs_ctx* c, int B, const cplx<R>* Ga, const cplx<R>* Gb, const R* phys_a, const R* phys_b,
                     cudaStream_t s) {
  RowTan2Params<R> p; p.Ga = Ga; p.Gb = Gb; p.H = (cplx<R>*)c->H; p.phys_a = phys_a; p.phys_b = phys_b;
  p.tw = (const cplx<R>*)c->tw; p.B = B;
  launch_step(c, B, k_row_tan2<R, N, XT>, dim3(B * (N / XT)), dim3(XT * 32), smem_row_tan2<R, N>(), s, p);
}

template <typename R, int N, int... ST>
void launch_col_tdj_sw(ecs_ctx* c, int B, int stage, cudaStream_t s, const ColTdjParams<R>& p,
                       std::integer_sequence<int, ST...>) {
  const int cols = B * Geomc<N>::K * 2;
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  ((stage == ST ? launch_step(c, B, k_col_tdj<R, N, ST>, g, bl, 0, s, p) : void()), ...);
}

template <typename R, int N>
void launch_col_tdj(ecs_ctx* c, int B, int stage, int produce, const cplx<R>* rec, const double* dT, double h,
                    double dscale, int nslot, cudaStream_t s) {
  ColTdjParams<R> p; p.H = (const cplx<R>*)c->H; p.Ga = (cplx<R>*)c->G; p.Gb = (cplx<R>*)c->Gx; p.D = (cplx<R>*)c->D;
  p.nslot = nslot; p.rec = rec; p.dT = dT; p.h = h; p.dscale = dscale; p.tw = (const cplx<R>*)c->tw;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B; p.produce = produce;
  launch_col_tdj_sw<R, N>(c, B, stage, s, p, std::make_integer_sequence<int, 5>{});
}

template <typename R, int N, int SCHEME, int... ST>
void launch_col_fxt_sw(ecs_ctx* c, int B, int stage, cudaStream_t s, const ColFxtParams<R>& p,
                       std::integer_sequence<int, ST...>) {
  const int cols = B * Geomc<N>::K * 2;
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  ((stage == ST ? launch_step(c, B, k_col_fxt<R, N, SCHEME, ST>, g, bl, 0, s, p) : void()), ...);
}

// Tangent column pass of the RK4 / Lawson-RK6 linearisation (kernels_fxl.cuh).
template <typename R, int N>
void launch_col_fxt(ecs_ctx* c, int B, int scheme, int stage, int produce, const cplx<R>* rec, const double* dT,
                    double h, double dscale, cudaStream_t s) {
  ColFxtParams<R> p{}; p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.D = (cplx<R>*)c->D;
  p.nslot = fxt_nslot(scheme); p.rec = rec; p.dT = dT; p.h = h; p.dscale = dscale; p.tw = (const cplx<R>*)c->tw;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B; p.produce = produce;
  if (scheme == FX_RK6) launch_col_fxt_sw<R, N, FX_RK6>(c, B, stage, s, p, std::make_integer_sequence<int, 9>{});
  else launch_col_fxt_sw<R, N, FX_RK4>(c, B, stage, s, p, std::make_integer_sequence<int, 5>{});
}

template <typename R, int N, int SCHEME, int... ST>
void launch_col_fxa_sw(ecs_ctx* c, int B, int stage, cudaStream_t s, const ColFxaParams<R>& p,
                       std::integer_sequence<int, ST...>) {
  const int cols = B * Geomc<N>::K * 2;
  const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
  ((stage == ST ? launch_step(c, B, k_col_fxa<R, N, SCHEME, ST>, g, bl, 0, s, p) : void()), ...);
}

// Adjoint column pass of the RK4 / Lawson-RK6 linearisation; stage S + 1 seeds a step.
template <typename R, int N>
void launch_col_fxa(ecs_ctx* c, int B, int scheme, int stage, const cplx<R>* rec, double h, cudaStream_t s) {
  ColFxaParams<R> p{}; p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.J = (cplx<R>*)c->D;
  p.nslot = fxa_nslot(scheme); p.rec = rec; p.hacc = c->hacc; p.h = h; p.tw = (const cplx<R>*)c->tw;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B;
  if (scheme == FX_RK6) launch_col_fxa_sw<R, N, FX_RK6>(c, B, stage, s, p, std::make_integer_sequence<int, 10>{});
  else launch_col_fxa_sw<R, N, FX_RK4>(c, B, stage, s, p, std::make_integer_sequence<int, 6>{});
}

inline int grid1d(long total, int threads = 256) {
  long g = (total + threads - 1) / threads;
  if (g > 148 * 32) g = 148 * 32;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace ecs

// ---------------------------------------------------------------------------
// per-(dtype, N) implementation
// ---------------------------------------------------------------------------
namespace ecs {

template <typename R, int N>
struct Impl {
  static constexpr int K = Geomc<N>::K, M = Geomc<N>::M;

  static int to_box(ecs_ctx* c, const R* fields, cplx<R>* box, int B, cudaStream_t s) {
    launch_row_to_box<R, N>(c, fields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, box, B, 2, s);
    return cuda_err(c, cudaGetLastError(), "to_box");
  }

  static int from_box(ecs_ctx* c, const cplx<R>* box, R* fields, int B, cudaStream_t s) {
    launch_col_from_box<R, N>(c, box, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, fields, nullptr, nullptr, B, 0, s);
    return cuda_err(c, cudaGetLastError(), "from_box");
  }

  static int dealias(ecs_ctx* c, const R* fields, R* out, int B, cudaStream_t s) {
    int st = to_box(c, fields, (cplx<R>*)c->V, B, s);
    if (st) return st;
    // mask[0,0] = False: drop the mean mode, then irfft2
    for (int b = 0; b < B; ++b)
      for (int ch = 0; ch < 2; ++ch) {
        cudaError_t e = cudaMemsetAsync((cplx<R>*)c->V + ((size_t)(b * 2 + ch) * K) * M, 0, sizeof(cplx<R>), s);
        if (e != cudaSuccess) return cuda_err(c, e, "dealias memset");
      }
    return from_box(c, (const cplx<R>*)c->V, out, B, s);
  }

  static int state_vel(ecs_ctx* c, const cplx<R>* fhat, cplx<R>* dfdt, int B, int diss, cudaStream_t s) {
    const long nbox = (long)B * 2 * K * M;
    ++c->launches; k_gather_box<R><<<grid1d(nbox), 256, 0, s>>>(fhat, (cplx<R>*)c->F, N, B);
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s);
    launch_row_rhs<R, N>(c, B, s);
    launch_col_rk4<R, N>(c, B, COL_PLAIN, 0, diss, s);
    const long nfull = (long)B * 2 * N * (N / 2 + 1);
    ++c->launches; k_scatter_box<R><<<grid1d(nfull), 256, 0, s>>>((const cplx<R>*)c->OUT, dfdt, N, B);
    return cuda_err(c, cudaGetLastError(), "state_vel");
  }

  // Calls go(W, DSM) with the chain shape for batch B and the exchange (dsm_default
  // unless ECS_CHAIN_DSMEM set it) as constants: 8 warps while B such clusters
  // fit on the device at once, else 16.
  template <typename F> static void chain_dispatch(const ecs_ctx* c, int B, bool dsm_default, F&& go) {
    using W8 = std::integral_constant<int, 8>;
    using W16 = std::integral_constant<int, 16>;
    const int w = c->chain_w ? c->chain_w : (B <= c->chain_res8 ? 8 : 16);
    const bool dsm = c->chain_dsm < 0 ? dsm_default : c->chain_dsm != 0;
    if (w == 8) {
      if (dsm) go(W8{}, std::true_type{}); else go(W8{}, std::false_type{});
    } else {
      if (dsm) go(W16{}, std::true_type{}); else go(W16{}, std::false_type{});
    }
  }
  // Whether a batch of B runs through a chain with batch range [minb, maxb] (maxb -1: the
  // 16-warp clusters the device holds at once).
  static bool chain_batch(const ecs_ctx* c, int B, int minb, int maxb) {
    if (N > 128) return false;
    const int hi = maxb < 0 ? c->chain_res16 : maxb;
    return B >= minb && B <= hi && (c->chain_res8 > 0 || c->chain_res16 > 0);
  }

  // Lawson-RK4 steps of the box states in c->F as one cluster-resident launch
  // (k_rk4_chain), after the COL_START pass; no inverse transforms after the last stage.
  static int rk4_chain(ecs_ctx* c, int B, long steps, cudaStream_t s) {
    if constexpr (N <= 128) {
      Rk4ChainParams<R> P{};
      ColParams<R>& p = P.col;
      p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.F = (cplx<R>*)c->F; p.A1 = (cplx<R>*)c->A1;
      p.K2 = (cplx<R>*)c->K2; p.OUT = (cplx<R>*)c->OUT; p.Etab = (const R*)c->Etab; p.ctl = c->ctl;
      p.fhat = (const cplx<R>*)c->fhat; p.tw = (const cplx<R>*)c->tw; p.nu = (R)c->nu; p.eta = (R)c->eta;
      p.B = B;
      RowParams<R>& q = P.row;
      q.G = (const cplx<R>*)c->G; q.H = (cplx<R>*)c->H; q.tw = (const cplx<R>*)c->tw;
      q.b0x = (R)c->b0x; q.b0y = (R)c->b0y; q.B = B;
      P.steps = steps; P.last_produce = 0;
      auto go = [&](auto w, auto dsm) {
        constexpr int W = decltype(w)::value;
        constexpr bool DSM = decltype(dsm)::value;
        launch_cluster(c, B, chain_cl<N, W>(), k_rk4_chain<R, N, W, DSM>, dim3(B * chain_cl<N, W>()), dim3(W * 32),
                       rk4_chain_smem<R, N, W, DSM>(), s, P);
      };
      chain_dispatch(c, B, true, go);
      return cuda_err(c, cudaGetLastError(), "rk4 chain");
    } else {
      (void)B; (void)steps; (void)s;
      return set_err(c, ECS_ERR_UNSUPPORTED, "rk4 chain: n > 128");
    }
  }

  // Lawson-RK4 over `steps` steps of the box state in c->F (ctl/Etab prepared).
  // Chunks of GS steps are captured once into a CUDA graph and replayed; batches
  // in the Lawson-RK4 chain range (chain_batch) run as one cluster-resident launch.
  static int integrate_rk4(ecs_ctx* c, int B, long steps, cudaStream_t s) {
    if (steps <= 0) return ECS_OK;
    constexpr int GS = 16;
    auto one_step = [&](cudaStream_t st_, bool last) {
      for (int st = 1; st <= 4; ++st) {
        launch_row_rhs<R, N>(c, B, st_);
        launch_col_rk4<R, N>(c, B, st, (st == 4 && last) ? 0 : 1, 0, st_);
      }
    };
    auto& gk = c->g4;
    if (steps > GS && !(gk.exec && gk.B == B)) {
      if (gk.exec) { cudaGraphExecDestroy(gk.exec); gk.exec = nullptr; }
      const long long l0 = c->launches;
      cudaGraph_t graph = nullptr;
      std::lock_guard<std::mutex> capture_guard(capture_mutex());   // no set-up of another context meanwhile
      cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int a = 0; a < GS; ++a) one_step(c->cap_stream, false);
        e = cudaStreamEndCapture(c->cap_stream, &graph);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&gk.exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) { gk.exec = nullptr; return cuda_err(c, e, "rk4 graph capture"); }
      gk.nodes = c->launches - l0;
      c->launches = l0;
      gk.B = B;
    }
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s);
    if (chain_batch(c, B, c->rk4chain_minb, c->rk4chain_maxb)) return rk4_chain(c, B, steps, s);
    long it = 0;
    while (steps - it > GS) {   // the final step (no inverse transforms) is launched directly
      cudaError_t e = cudaGraphLaunch(gk.exec, s);
      if (e != cudaSuccess) return cuda_err(c, e, "rk4 graph launch");
      c->launches += gk.nodes;
      it += GS;
    }
    for (; it < steps; ++it) one_step(s, it == steps - 1);
    return cuda_err(c, cudaGetLastError(), "integrate_rk4");
  }

  // Fixed-step RK4 / Lawson-RK6 / TDRK4 over `steps` steps from slot X_F of S43
  // (h and e from fx_setup); 16-step CUDA graphs per scheme.
  static int integrate_fx(ecs_ctx* c, int scheme, int B, long steps, cudaStream_t s) {
    PlainOrder plain_order(c);
    if (steps <= 0) return ECS_OK;
    constexpr int GS = 16;
    R* phys = nullptr;
    const long pstride = (long)N * NPH * N;
    if (scheme == FX_TD4) {
      const int st = grow(c, &c->fxphys, &c->fxphys_bytes, (size_t)B * pstride * sizeof(R));
      if (st) return st;
      phys = (R*)c->fxphys;
    }
    const int nst = scheme == FX_RK6 ? 8 : 4;
    auto one_step = [&](cudaStream_t st_, bool last) {
      for (int q = 1; q <= nst; ++q) {
        const int produce = (q == nst && last) ? 0 : 1;
        if (scheme == FX_TD4 && (q == 2 || q == 4)) launch_row_tan<R, N>(c, B, phys, st_, pstride);   // jac(., k)
        else launch_row_rhs<R, N>(c, B, st_, nullptr, phys, pstride);
        launch_col_fx<R, N>(c, B, scheme, q, produce, st_);
      }
    };
    auto& gk = c->gfx[scheme];
    if (steps > GS && !(gk.exec && gk.B == B && gk.phys == (void*)phys)) {
      if (gk.exec) { cudaGraphExecDestroy(gk.exec); gk.exec = nullptr; }
      const long long l0 = c->launches;
      cudaGraph_t graph = nullptr;
      std::lock_guard<std::mutex> capture_guard(capture_mutex());   // no set-up of another context meanwhile
      cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int a = 0; a < GS; ++a) one_step(c->cap_stream, false);
        e = cudaStreamEndCapture(c->cap_stream, &graph);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&gk.exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) { gk.exec = nullptr; return cuda_err(c, e, "fixed-step graph capture"); }
      gk.nodes = c->launches - l0;
      c->launches = l0;
      gk.B = B; gk.phys = phys;
    }
    launch_col_fx<R, N>(c, B, scheme, 0, 1, s);
    long it = 0;
    while (steps - it > GS) {
      cudaError_t e = cudaGraphLaunch(gk.exec, s);
      if (e != cudaSuccess) return cuda_err(c, e, "fixed-step graph launch");
      c->launches += gk.nodes;
      it += GS;
    }
    for (; it < steps; ++it) one_step(s, it == steps - 1);
    return cuda_err(c, cudaGetLastError(), "integrate_fx");
  }

  // modes whose right-hand side (or unmasked integrating factor) leaves the modes outside the box unchanged
  static bool carry_mode(int mode) {
    return mode == ECS_MODE_LAWSON_RK43 || mode == ECS_MODE_RK4 || mode == ECS_MODE_TDRK4;
  }

  static int fx_scheme(int mode) {
    return mode == ECS_MODE_RK4 ? (int)FX_RK4 : mode == ECS_MODE_LAWSON_RK6 ? (int)FX_RK6 : (int)FX_TD4;
  }

  // Fixed-step integration of full rfft2 states f_hat [B][2][N][N/2+1] in place
  // (timestepping.py rk4 / lawson_rk4 / lawson_rk6 / tdrk4 with the v_fn,
  // L_diag and mask of mismatch_RPO's mode).
  static int integrate_mode(ecs_ctx* c, int mode, cplx<R>* fhat, double t, int steps, int B, cudaStream_t s) {
    if (mode == ECS_MODE_LAWSON_RK4) return lawson_rk4(c, fhat, t, steps, B, s);
    if (mode != ECS_MODE_RK4 && mode != ECS_MODE_LAWSON_RK6 && mode != ECS_MODE_TDRK4)
      return set_err(c, ECS_ERR_BAD_MODE, "ecs_integrate: fixed-step modes only");
    const long VEC = 2L * K * M;
    ++c->launches; k_fill<<<1, 256, 0, s>>>(c->Tbuf, t, B);
    ++c->launches; k_gather_box<R><<<grid1d((long)B * VEC), 256, 0, s>>>(fhat, (cplx<R>*)c->F, N, B);
    cudaError_t e = cudaMemcpy2DAsync((cplx<R>*)c->S43 + X_F * VEC, S_NSLOT * VEC * sizeof(cplx<R>), c->F,
                                      VEC * sizeof(cplx<R>), VEC * sizeof(cplx<R>), B, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_err(c, e, "integrate");
    ++c->launches;
    k_fx_setup<R><<<grid1d((long)B * VEC), 256, 0, s>>>(c->Tbuf, 1, steps, 6, c->ctl, (R*)c->Etab, N, c->nu, c->eta, B);
    int st = integrate_fx(c, fx_scheme(mode), B, steps, s);
    if (st) return st;
    e = cudaMemcpy2DAsync(c->F, VEC * sizeof(cplx<R>), (const cplx<R>*)c->S43 + X_F * VEC,
                          S_NSLOT * VEC * sizeof(cplx<R>), VEC * sizeof(cplx<R>), B, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_err(c, e, "integrate");
    const long nfull = (long)B * 2 * N * (N / 2 + 1);
    ++c->launches;
    if (carry_mode(mode)) k_scatter_box_keep<R><<<grid1d(nfull), 256, 0, s>>>((const cplx<R>*)c->F, fhat, N, B);
    else k_scatter_box<R><<<grid1d(nfull), 256, 0, s>>>((const cplx<R>*)c->F, fhat, N, B);
    return cuda_err(c, cudaGetLastError(), "integrate");
  }

  static int recurrence(ecs_ctx* c, const cplx<R>* fs, int S, double* dist, cudaStream_t s) {
    const long len = 2L * N * (N / 2 + 1);
    ++c->launches; k_recurrence<R><<<dim3(S, S), 256, 0, s>>>(fs, S, len, dist);
    return cuda_err(c, cudaGetLastError(), "recurrence");
  }

  static int rk4_setup(ecs_ctx* c, const double* T, int nc, int ms, int B, cudaStream_t s) {
    const long tot = (long)B * 2 * K * M;
    ++c->launches; k_rk4_setup<R><<<grid1d(tot), 256, 0, s>>>(T, nc, ms, c->ctl, (R*)c->Etab, N, c->nu, c->eta, B);
    return cuda_err(c, cudaGetLastError(), "rk4_setup");
  }

  static int lawson_rk4(ecs_ctx* c, cplx<R>* fhat, double t, int steps, int B, cudaStream_t s) {
    ++c->launches; k_fill<<<1, 256, 0, s>>>(c->Tbuf, t, B);
    int st = rk4_setup(c, c->Tbuf, 1, steps, B, s);
    if (st) return st;
    const long nbox = (long)B * 2 * K * M;
    ++c->launches; k_gather_box<R><<<grid1d(nbox), 256, 0, s>>>(fhat, (cplx<R>*)c->F, N, B);
    st = integrate_rk4(c, B, steps, s);
    if (st) return st;
    const long nfull = (long)B * 2 * N * (N / 2 + 1);
    ++c->launches; k_scatter_box<R><<<grid1d(nfull), 256, 0, s>>>((const cplx<R>*)c->F, fhat, N, B);
    return cuda_err(c, cudaGetLastError(), "lawson_rk4");
  }

  // Adaptive Lawson-RK4(3) of the box states in S43[b][S_X0] (timestepping.py:151-335).
  // Returns after all candidates completed or the attempt cap was reached.
  static int rk43_solve(ecs_ctx* c, const ecs_shoot_cfg* cfg, const double* T, int B, cudaStream_t s,
                        cplx<R>* rec = nullptr, double* rec_h = nullptr, int* rec_acc = nullptr, int cap = 0,
                        bool launch = true) {
    PlainOrder plain_order(c);
    const long amax = (long)cfg->checkpoints * cfg->max_steps_per_checkpoint;
    if (amax <= 0) return set_err(c, ECS_ERR_INVALID, "checkpoints * max_steps_per_checkpoint must be > 0");
    ++c->launches; k_rk43_setup<<<(B + 127) / 128, 128, 0, s>>>(T, cfg->h0, c->ctl, B);
    launch_col_rk43<R, N>(c, B, R43_START, s);
    launch_row_rhs<R, N>(c, B, s, c->ctl);
    launch_col_rk43<R, N>(c, B, R43_INIT, s);
    if (launch && chain_batch(c, B, c->rk43chain_minb, c->rk43chain_maxb)) {
      // the attempts as one cluster-resident launch, no host round trip (k_rk43_chain)
      if constexpr (N <= 128) {
        Rk43ChainParams<R> P{};
        Col43Params<R>& q = P.col;
        q.H = (const cplx<R>*)c->H; q.G = (cplx<R>*)c->G; q.S = (cplx<R>*)c->S43; q.ctl = c->ctl;
        q.fhat = (const cplx<R>*)c->fhat; q.tw = (const cplx<R>*)c->tw; q.rec = rec; q.cap = cap;
        q.nu = (R)c->nu; q.eta = (R)c->eta; q.B = B;
        RowParams<R>& r = P.row;
        r.G = (const cplx<R>*)c->G; r.H = (cplx<R>*)c->H; r.tw = (const cplx<R>*)c->tw; r.ctl = c->ctl;
        r.b0x = (R)c->b0x; r.b0y = (R)c->b0y; r.B = B;
        P.atol = cfg->atol; P.rec_h = rec_h; P.rec_acc = rec_acc; P.amax = amax;
        if (c->chain_w == 8 || (c->chain_w == 0 && B <= c->chain_res8))
          launch_cluster(c, B, chain_cl<N, 8>(), k_rk43_chain<R, N, 8>, dim3(B * chain_cl<N, 8>()), dim3(8 * 32),
                         rk43_chain_smem<R, N, 8>(), s, P);
        else
          launch_cluster(c, B, chain_cl<N, 16>(), k_rk43_chain<R, N, 16>, dim3(B * chain_cl<N, 16>()), dim3(16 * 32),
                         rk43_chain_smem<R, N, 16>(), s, P);
        const long nbox = (long)B * 2 * K * M;
        ++c->launches; k_rk43_resolve<R><<<grid1d(nbox), 256, 0, s>>>((cplx<R>*)c->S43, c->ctl, (cplx<R>*)c->F, N, B);
        return cuda_err(c, cudaGetLastError(), "rk43 chain");
      }
    }
    // one attempt = 5 column + 4 row + 1 error launches; a chunk of GA attempts is
    // captured once into a CUDA graph (all per-attempt data is read from the
    // device control block, so the same graph replays every chunk)
    auto attempt = [&](cudaStream_t st_) {
      launch_col_rk43<R, N>(c, B, R43_A, st_, rec, cap);
      for (int st = R43_B; st <= R43_E; ++st) {
        launch_row_rhs<R, N>(c, B, st_, c->ctl);
        launch_col_rk43<R, N>(c, B, st, st_, rec, cap);
      }
      launch_row_err<R, N>(c, B, cfg->atol, st_, rec_h, rec_acc, cap);
    };
    constexpr int GA = 16;
    auto& gk = c->g43;
    const bool same = gk.exec && gk.B == B && gk.atol == cfg->atol && gk.rec == (void*)rec && gk.rec_h == rec_h &&
                      gk.rec_acc == rec_acc && gk.cap == cap && gk.G == c->G && gk.H == c->H;
    if (!same && amax >= GA) {
      if (gk.exec) { cudaGraphExecDestroy(gk.exec); gk.exec = nullptr; }
      const long long l0 = c->launches;
      cudaGraph_t graph = nullptr;
      std::lock_guard<std::mutex> capture_guard(capture_mutex());   // no set-up of another context meanwhile
      cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int a = 0; a < GA; ++a) attempt(c->cap_stream);
        e = cudaStreamEndCapture(c->cap_stream, &graph);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&gk.exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) { gk.exec = nullptr; return cuda_err(c, e, "rk43 graph capture"); }
      gk.nodes = c->launches - l0;
      c->launches = l0;
      gk.B = B; gk.atol = cfg->atol; gk.rec = rec; gk.rec_h = rec_h; gk.rec_acc = rec_acc; gk.cap = cap;
      gk.G = c->G; gk.H = c->H;
    }
    if (!launch) return ECS_OK;   // set-up and graph only (the pipelined linearisation drives the chunks)
    long a = 0;
    while (a < amax) {
      if (gk.exec && amax - a >= GA) {
        cudaError_t e = cudaGraphLaunch(gk.exec, s);
        if (e != cudaSuccess) return cuda_err(c, e, "rk43 graph launch");
        c->launches += gk.nodes;
        a += GA;
      } else {
        attempt(s);
        a += 1;
        if (a % GA != 0 && a != amax) continue;
      }
      ++c->launches; k_count_done<<<1, 32, 0, s>>>(c->ctl, c->dcount, B);
      cudaError_t e = cudaMemcpyAsync(c->hcount, c->dcount, sizeof(int), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return cuda_err(c, e, "rk43 completion check");
      if (*c->hcount == B) break;
    }
    const long nbox = (long)B * 2 * K * M;
    ++c->launches; k_rk43_resolve<R><<<grid1d(nbox), 256, 0, s>>>((cplx<R>*)c->S43, c->ctl, (cplx<R>*)c->F, N, B);
    return cuda_err(c, cudaGetLastError(), "rk43_solve");
  }

  // Forward shooting map + symmetries + residual (objective_RPO / loss_RPO).
  static int shoot(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                   R* out_fields, double* loss, ecs_info* info, int B, cudaStream_t s) {
    const bool rk43 = cfg->mode == ECS_MODE_LAWSON_RK43;
    const bool fx = cfg->mode == ECS_MODE_RK4 || cfg->mode == ECS_MODE_LAWSON_RK6 || cfg->mode == ECS_MODE_TDRK4;
    if (cfg->mode != ECS_MODE_LAWSON_RK4 && !rk43 && !fx)
      return set_err(c, ECS_ERR_BAD_MODE, "unknown integration mode");   // loss_functions.py:86-88
    int st;
    const long VEC = 2L * K * M;
    // modes outside the box are carried unchanged by the adaptive stepper (unmasked
    // integrating factor) and by RK4 / TDRK4 (masked right-hand side, no factor)
    const bool carry = carry_mode(cfg->mode);
    if (fx) {
      if (cfg->num_checkpoints <= 0 || cfg->ministeps <= 0) return set_err(c, ECS_ERR_INVALID, "steps must be > 0");
      const int scheme = fx_scheme(cfg->mode);
      launch_row_to_box<R, N>(c, fields, (cplx<R>*)c->H, B, s);
      launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->S43 + X_F * VEC, B, 2, s, S_NSLOT * VEC);
      launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->V, B, 2, s);
      ++c->launches;
      k_fx_setup<R><<<grid1d((long)B * VEC), 256, 0, s>>>(T, cfg->num_checkpoints, cfg->ministeps, 6, c->ctl,
                                                           (R*)c->Etab, N, c->nu, c->eta, B);
      st = integrate_fx(c, scheme, B, (long)cfg->num_checkpoints * cfg->ministeps, s);
      if (st) return st;
      const cudaError_t e = cudaMemcpy2DAsync(c->F, VEC * sizeof(cplx<R>), (const cplx<R>*)c->S43 + X_F * VEC,
                                              S_NSLOT * VEC * sizeof(cplx<R>), VEC * sizeof(cplx<R>), B,
                                              cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return cuda_err(c, e, "fixed-step result");
    } else if (!rk43) {
      if (cfg->num_checkpoints <= 0 || cfg->ministeps <= 0) return set_err(c, ECS_ERR_INVALID, "steps must be > 0");
      st = to_box(c, fields, (cplx<R>*)c->F, B, s);
      if (st) return st;
      st = rk4_setup(c, T, cfg->num_checkpoints, cfg->ministeps, B, s);
      if (st) return st;
      st = integrate_rk4(c, B, (long)cfg->num_checkpoints * cfg->ministeps, s);
      if (st) return st;
    } else {
      launch_row_to_box<R, N>(c, fields, (cplx<R>*)c->H, B, s);
      launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->S43 + S_X0 * VEC, B, 2, s, S_NSLOT * VEC);
      launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->V, B, 2, s);
      st = rk43_solve(c, cfg, T, B, s);
      if (st) return st;
    }
    R* out = out_fields ? out_fields : (R*)c->fields_tmp;
    if (carry) {   // fields - irfft2(box(fields)): the modes outside the box
      launch_col_from_box<R, N>(c, (const cplx<R>*)c->V, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
      launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, (R*)c->fields_tmp2, fields, nullptr, B, 1, s);
    }
    launch_col_from_box<R, N>(c, (const cplx<R>*)c->F, (cplx<R>*)c->G, B, sx, cfg->shift_reflect_ny, cfg->rot, 1, 0, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, out, fields, nullptr, B, 1, s);
    if (carry) {
      const int odd = (cfg->shift_reflect_ny % 2 + 2) % 2 == 1;
      ++c->launches; k_sub_sym_phys<R><<<grid1d((long)B * 2 * N * N), 256, 0, s>>>(out, (const R*)c->fields_tmp2, odd, cfg->rot, N, B);
    }
    if (loss) {
      ++c->launches; k_rowsq<R><<<B * N, 32, 0, s>>>(out, c->rowsq, N);
      ++c->launches; k_reduce_rows<<<(B + 127) / 128, 128, 0, s>>>(c->rowsq, loss, N, B, 1.0 / (2.0 * N * N));
    }
    st = cuda_err(c, cudaGetLastError(), "shoot");
    if (st) return st;
    if (info) {
      if (rk43) {
        std::vector<StepCtl> h(B);
        cudaError_t e = cudaMemcpyAsync(h.data(), c->ctl, sizeof(StepCtl) * B, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_err(c, e, "info readback");
        for (int b = 0; b < B; ++b) {
          info[b].completed = h[b].done; info[b].s = h[b].s; info[b].accepted = h[b].accepted;
          info[b].rejected = h[b].rejected; info[b].fevals = h[b].fevals;
        }
      } else {
        const int steps = cfg->num_checkpoints * cfg->ministeps;
        for (int b = 0; b < B; ++b) {
          info[b].completed = 1; info[b].s = 1.0; info[b].accepted = steps; info[b].rejected = 0;
          info[b].fevals = 4 * steps;
        }
      }
    }
    return ECS_OK;
  }

  // Record `steps` Lawson-RK4 steps of the box state in c->F (batch 1) into rec
  // (Q_NREC vectors per step); ctl/Etab must hold the step size of the call.
  static void record_rk4_segment(ecs_ctx* c, cplx<R>* rec, long steps, cudaStream_t s) {
    const size_t VEC = 2UL * K * M;
    launch_col_rk4<R, N>(c, 1, COL_START, 1, 0, s);
    for (long it = 0; it < steps; ++it) {
      cplx<R>* rs = rec + (size_t)it * Q_NREC * VEC;
      for (int k = 1; k <= 4; ++k) {
        launch_row_rhs<R, N>(c, 1, s);
        launch_col_rk4<R, N>(c, 1, k, (k == 4 && it == steps - 1) ? 0 : 1, 0, s, rs, 0);
      }
    }
  }

  // Lawson-RK4 segment [a0, a0+cnt) of the current linearisation: its record
  // (recomputed from the checkpoint when the linearisation is segmented).
  static const cplx<R>* rk4_segment_record(ecs_ctx* c, long a0, long cnt, cudaStream_t s, void* buf = nullptr) {
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    if (!L.seg) return (const cplx<R>*)L.rec + (size_t)a0 * Q_NREC * VEC;
    cplx<R>* dst = (cplx<R>*)(buf ? buf : L.rec);
    rk4_setup(c, L.dT, L.cfg.num_checkpoints, L.cfg.ministeps, 1, s);
    cudaMemcpyAsync(c->F, (cplx<R>*)L.ckpt + (size_t)(a0 / L.seg) * VEC, vb, cudaMemcpyDeviceToDevice, s);
    record_rk4_segment(c, dst, cnt, s);
    return dst;
  }

  // ---------------------------------------------------------------------
  // Linearisation: primal solve of one candidate with its trajectory record,
  // plus the stop-gradient phase fields vt, vx (loss_functions.py:113-130).
  // ---------------------------------------------------------------------
  // Linearisation prologue: scalars, box(f0), the phase fields vt and vx.
  static int lin_prologue(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                          cudaStream_t s) {
    auto& L = c->lin;
    L.valid = 0;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>), fb = 2UL * N * N * sizeof(R);
    (void)VEC;
    int st = ECS_OK;
    size_t dummy = 0;
    if (!L.phi) {
      L.phi = dev_alloc(c, vb, &st); L.f0box = dev_alloc(c, vb, &st);
      L.vt = dev_alloc(c, fb, &st); L.vx = dev_alloc(c, fb, &st);
      L.dsx = (double*)dev_alloc(c, 64, &st); L.dT = (double*)dev_alloc(c, 64, &st);
      if (st) return st;
    }
    (void)dummy;
    double hT = 0, hsx = 0;
    cudaError_t e = cudaMemcpyAsync(&hT, T, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&hsx, sx, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.dsx, sx, sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(L.dT, T, sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_err(c, e, "linearize scalars");
    L.T = hT; L.sx = hsx; L.cfg = *cfg; L.mode = cfg->mode;
    // f0 box and the phase fields
    st = to_box(c, fields, (cplx<R>*)L.f0box, 1, s);
    if (st) return st;
    cudaMemcpyAsync(c->F, L.f0box, vb, cudaMemcpyDeviceToDevice, s);
    launch_col_rk4<R, N>(c, 1, COL_START, 1, 0, s);
    launch_row_rhs<R, N>(c, 1, s);
    launch_col_rk4<R, N>(c, 1, COL_PLAIN, 0, 1, s);
    st = from_box(c, (const cplx<R>*)c->OUT, (R*)L.vt, 1, s);
    if (st) return st;
    launch_col_from_box<R, N>(c, (const cplx<R>*)L.f0box, (cplx<R>*)c->G, 1, nullptr, 0, 0, 0, 1, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, (R*)L.vx, nullptr, nullptr, 1, 0, s);
    return cuda_err(c, cudaGetLastError(), "linearize prologue");
  }

  // Lawson-RK4(3) record buffers for `cap` attempts and the start state.
  static int lin43_alloc(ecs_ctx* c, const ecs_shoot_cfg* cfg, cudaStream_t s) {
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const long cap = (long)cfg->checkpoints * cfg->max_steps_per_checkpoint;
    if (cap <= 0) return set_err(c, ECS_ERR_INVALID, "checkpoints * max_steps_per_checkpoint must be > 0");
    int st = grow(c, &L.rec, &L.rec_bytes, (size_t)cap * RR_NREC * vb);
    if (st) return st;
    if ((size_t)cap > L.cap) {
      if (L.rec_h) { cudaFree(L.rec_h); cudaFree(L.rec_acc); }
      if (cudaMalloc(&L.rec_h, cap * sizeof(double)) != cudaSuccess || cudaMalloc(&L.rec_acc, cap * sizeof(int)) != cudaSuccess)
        return set_err(c, ECS_ERR_OOM, "record allocation");
      L.cap = cap;
    }
    cudaMemcpyAsync((cplx<R>*)c->S43 + S_X0 * VEC, L.f0box, vb, cudaMemcpyDeviceToDevice, s);
    return cuda_err(c, cudaGetLastError(), "record allocation");
  }

  // TDRK4 linearisation (batch 1): the forward solve recording per step the
  // start state, k1, a1, f_temp, k2, a2 (TR_NREC box vectors).
  static int linearize_td(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                          R* out_fields, ecs_info* info, cudaStream_t s) {
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const long steps = (long)cfg->num_checkpoints * cfg->ministeps;
    if (steps <= 0) return set_err(c, ECS_ERR_INVALID, "steps must be > 0");
    int st = lin_prologue(c, cfg, fields, T, sx, s);
    if (!st) st = grow(c, &L.rec, &L.rec_bytes, (size_t)steps * TR_NREC * vb);
    if (!st) st = grow(c, &c->fxphys, &c->fxphys_bytes, (size_t)N * NPH * N * sizeof(R));
    if (st) return st;
    cudaMemcpyAsync((cplx<R>*)c->S43 + X_F * VEC, L.f0box, vb, cudaMemcpyDeviceToDevice, s);
    ++c->launches;
    k_fx_setup<R><<<grid1d((long)VEC), 256, 0, s>>>(T, cfg->num_checkpoints, cfg->ministeps, 6, c->ctl, (R*)c->Etab, N,
                                                    c->nu, c->eta, 1);
    R* phys = (R*)c->fxphys;
    cplx<R>* rec = (cplx<R>*)L.rec;
    launch_col_fx<R, N>(c, 1, FX_TD4, 0, 1, s);
    for (long it = 0; it < steps; ++it) {
      cplx<R>* rs = rec + (size_t)it * TR_NREC * VEC;
      for (int q = 1; q <= 4; ++q) {
        if (q == 2 || q == 4) launch_row_tan<R, N>(c, 1, phys, s, 0);
        else launch_row_rhs<R, N>(c, 1, s, nullptr, phys, 0);
        launch_col_fx<R, N>(c, 1, FX_TD4, q, (q == 4 && it == steps - 1) ? 0 : 1, s, rs);
      }
    }
    cudaMemcpyAsync(L.phi, (cplx<R>*)c->S43 + X_F * VEC, vb, cudaMemcpyDeviceToDevice, s);
    L.seg = 0;
    L.nrec = steps;
    L.h = (double)(R)((L.T / (double)cfg->num_checkpoints) / (double)cfg->ministeps);
    L.acc.clear(); L.hs.clear();
    if (info) { info->completed = 1; info->s = 1.0; info->accepted = (int)steps; info->rejected = 0; info->fevals = (int)(4 * steps); }
    if (out_fields) {
      st = residual(c, cfg, fields, (const cplx<R>*)L.phi, (const cplx<R>*)L.f0box, L.dsx, 1, out_fields, s, 1);
      if (st) return st;
    }
    L.valid = 1;
    return cuda_err(c, cudaGetLastError(), "linearize (TDRK4)");
  }

  // TDRK4 JVP sweep for B tangents (see kernels_fx.cuh for the tangent algebra):
  // per step the primal's f and f_temp (with the mean field) and k1, k2 (without)
  // are regenerated in chunks of steps and shared by the batch.
  static int jvp_td(ecs_ctx* c, const R* dfields, const double* dT, const double* dsx, R* out, double* odT,
                    double* odsx, int B, cudaStream_t s) {
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const int nslot = (int)DT_NSLOT;
    int st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = grow(c, &c->Gx, &c->Gx_bytes, (size_t)B * NG * K * N * sizeof(cplx<R>));
    if (!st) st = ensure_regen(c);
    if (st) return st;
    launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->D + (size_t)DT_F * VEC, B, 2, s, (long)nslot * VEC);
    const long steps = L.nrec;
    const long ci = (long)chunk_items(c);
    const long CS = std::max(1L, std::min(64L, ci / 4));   // steps per regeneration chunk (4 items each)
    // items: per chunk, the states [f, f_temp] of its steps, then the derivatives [k1, k2]
    std::vector<long> items;
    items.reserve((size_t)(4 * steps));
    for (long a0 = 0; a0 < steps; a0 += CS) {
      const long cnt = std::min(CS, steps - a0);
      for (long it = a0; it < a0 + cnt; ++it) { items.push_back(it * TR_NREC + TR_F); items.push_back(it * TR_NREC + TR_FT); }
      for (long it = a0; it < a0 + cnt; ++it) { items.push_back(it * TR_NREC + TR_K1); items.push_back(it * TR_NREC + TR_K2); }
    }
    st = upload_items(c, items, s);
    if (st) return st;
    const cplx<R>* rec = (const cplx<R>*)L.rec;
    const double dscale = 1.0 / ((double)L.cfg.num_checkpoints * (double)L.cfg.ministeps);
    const size_t pst = (size_t)N * NPH * N;
    const cplx<R>* Ga = (const cplx<R>*)c->G;
    const cplx<R>* Gb = (const cplx<R>*)c->Gx;
    launch_col_tdj<R, N>(c, B, 0, 1, rec, dT, L.h, dscale, nslot, s);
    for (long a0 = 0; a0 < steps; a0 += CS) {
      const long cnt = std::min(CS, steps - a0);
      R* P = (R*)c->Phys;
      launch_regen<R, N>(c, rec, c->items + 4 * a0, (int)(2 * cnt), s, P, true);
      launch_regen<R, N>(c, rec, c->items + 4 * a0 + 2 * cnt, (int)(2 * cnt), s, P + 2 * cnt * pst, false);
      for (long it = a0; it < a0 + cnt; ++it) {
        const cplx<R>* ra = rec + (size_t)it * TR_NREC * VEC;
        const R* pf = P + (size_t)(2 * (it - a0)) * pst;
        const R* pft = pf + pst;
        const R* pk1 = P + (size_t)(2 * cnt + 2 * (it - a0)) * pst;
        const R* pk2 = pk1 + pst;
        launch_row_tan<R, N>(c, B, pf, s);                        // N'(f) df
        launch_col_tdj<R, N>(c, B, 1, 1, ra, dT, L.h, dscale, nslot, s);
        launch_row_tan2<R, N>(c, B, Ga, Gb, pf, pk1, s);          // N'(f) dk1 + N'(k1) df
        launch_col_tdj<R, N>(c, B, 2, 1, ra, dT, L.h, dscale, nslot, s);
        launch_row_tan<R, N>(c, B, pft, s);                       // N'(f_temp) dft
        launch_col_tdj<R, N>(c, B, 3, 1, ra, dT, L.h, dscale, nslot, s);
        launch_row_tan2<R, N>(c, B, Ga, Gb, pft, pk2, s);         // N'(f_temp) dk2 + N'(k2) dft
        launch_col_tdj<R, N>(c, B, 4, it == steps - 1 ? 0 : 1, ra, dT, L.h, dscale, nslot, s);
      }
    }
    return jvp_finish(c, dfields, dsx, out, odT, odsx, B, s);
  }

  // ---------------------------------------------------------------------
  // Classic RK4 and Lawson-RK6 (kernels_fxl.cuh): linearisation = the batch-1
  // forward solve with a record per step [f0, k_1..k_S, x_2..x_S]; the JVP
  // sweep runs the tangent stages forward over it, the VJP sweep the adjoint
  // stages backward, both with the primal physical fields of every stage input
  // regenerated in chunks from the record and shared by the batch.
  // ---------------------------------------------------------------------
  static bool fxl_mode(int mode) { return mode == ECS_MODE_RK4 || mode == ECS_MODE_LAWSON_RK6; }

  static int linearize_fxl(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                           R* out_fields, ecs_info* info, cudaStream_t s) {
    auto& L = c->lin;
    const int scheme = fx_scheme(cfg->mode), S = fxl_stages(scheme), NR = fxr_n(scheme);
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const long steps = (long)cfg->num_checkpoints * cfg->ministeps;
    if (steps <= 0) return set_err(c, ECS_ERR_INVALID, "steps must be > 0");
    int st = lin_prologue(c, cfg, fields, T, sx, s);
    if (!st) st = grow(c, &L.rec, &L.rec_bytes, (size_t)steps * NR * vb);
    if (st) return st;
    PlainOrder plain_order(c);
    cudaMemcpyAsync((cplx<R>*)c->S43 + X_F * VEC, L.f0box, vb, cudaMemcpyDeviceToDevice, s);
    ++c->launches;
    k_fx_setup<R><<<grid1d((long)VEC), 256, 0, s>>>(T, cfg->num_checkpoints, cfg->ministeps, 6, c->ctl, (R*)c->Etab, N,
                                                    c->nu, c->eta, 1);
    cplx<R>* rec = (cplx<R>*)L.rec;
    launch_col_fx<R, N>(c, 1, scheme, 0, 1, s);
    for (long it = 0; it < steps; ++it) {
      cplx<R>* rs = rec + (size_t)it * NR * VEC;
      for (int q = 1; q <= S; ++q) {
        launch_row_rhs<R, N>(c, 1, s);
        launch_col_fx<R, N>(c, 1, scheme, q, (q == S && it == steps - 1) ? 0 : 1, s, rs);
      }
    }
    cudaMemcpyAsync(L.phi, (cplx<R>*)c->S43 + X_F * VEC, vb, cudaMemcpyDeviceToDevice, s);
    L.seg = 0;
    L.nrec = steps;
    L.h = (double)(R)((L.T / (double)cfg->num_checkpoints) / (double)cfg->ministeps);
    L.acc.clear(); L.hs.clear();
    if (info) { info->completed = 1; info->s = 1.0; info->accepted = (int)steps; info->rejected = 0; info->fevals = (int)(S * steps); }
    if (out_fields) {
      st = residual(c, cfg, fields, (const cplx<R>*)L.phi, (const cplx<R>*)L.f0box, L.dsx, 1, out_fields, s, 1);
      if (st) return st;
    }
    L.valid = 1;
    return cuda_err(c, cudaGetLastError(), "linearize (RK4 / Lawson-RK6)");
  }

  // Regeneration plan of the fixed-step linearisation: per step, the S stage inputs.
  static std::vector<long> fxl_items(int scheme, long steps) {
    const int S = fxl_stages(scheme), NR = fxr_n(scheme);
    std::vector<long> items;
    items.reserve((size_t)(S * steps));
    for (long it = 0; it < steps; ++it)
      for (int q = 1; q <= S; ++q) items.push_back(it * NR + (q == 1 ? fxr_f() : fxr_x(scheme, q)));
    return items;
  }

  static int jvp_fxl(ecs_ctx* c, const R* dfields, const double* dT, const double* dsx, R* out, double* odT,
                     double* odsx, int B, cudaStream_t s) {
    auto& L = c->lin;
    const int scheme = fx_scheme(L.mode), S = fxl_stages(scheme), NR = fxr_n(scheme), nslot = fxt_nslot(scheme);
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    int st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = ensure_regen(c);
    if (st) return st;
    launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->D + (size_t)FT_F * VEC, B, 2, s, (long)nslot * VEC);
    const long steps = L.nrec;
    const std::vector<long> items = fxl_items(scheme, steps);
    st = upload_items(c, items, s);
    if (st) return st;
    const long ci = (long)chunk_items(c);
    long chunk_lo = -1;
    const cplx<R>* rec = (const cplx<R>*)L.rec;
    auto phys_of = [&](long item) -> const R* {
      if (chunk_lo < 0 || item < chunk_lo || item >= chunk_lo + ci) {
        chunk_lo = item;
        const long cnt = std::min<long>(ci, (long)items.size() - item);
        launch_regen<R, N>(c, rec, c->items + item, (int)cnt, s);
      }
      return (const R*)c->Phys + (size_t)(item - chunk_lo) * N * NPH * N;
    };
    const double dscale = 1.0 / ((double)L.cfg.num_checkpoints * (double)L.cfg.ministeps);
    launch_col_fxt<R, N>(c, B, scheme, 0, 1, rec, dT, L.h, dscale, s);
    for (long it = 0; it < steps; ++it) {
      const cplx<R>* ra = rec + (size_t)it * NR * VEC;
      for (int q = 1; q <= S; ++q) {
        launch_row_tan<R, N>(c, B, phys_of(it * S + q - 1), s);
        launch_col_fxt<R, N>(c, B, scheme, q, (q == S && it == steps - 1) ? 0 : 1, ra, dT, L.h, dscale, s);
      }
    }
    return jvp_finish(c, dfields, dsx, out, odT, odsx, B, s);
  }

  static int vjp_fxl_sweep(ecs_ctx* c, int B, cudaStream_t s) {
    auto& L = c->lin;
    const int scheme = fx_scheme(L.mode), S = fxl_stages(scheme), NR = fxr_n(scheme);
    const size_t VEC = 2UL * K * M;
    const long steps = L.nrec;
    const std::vector<long> items = fxl_items(scheme, steps);
    int st = upload_items(c, items, s);
    if (st) return st;
    const long ci = (long)chunk_items(c);
    long chunk_lo = -1;
    const cplx<R>* rec = (const cplx<R>*)L.rec;
    auto phys_of = [&](long item) -> const R* {   // chunks end at the requested item (reverse sweep)
      if (chunk_lo < 0 || item < chunk_lo || item >= chunk_lo + ci) {
        chunk_lo = std::max<long>(0, item - ci + 1);
        const long cnt = std::min<long>(ci, (long)items.size() - chunk_lo);
        launch_regen<R, N>(c, rec, c->items + chunk_lo, (int)cnt, s);
      }
      return (const R*)c->Phys + (size_t)(item - chunk_lo) * N * NPH * N;
    };
    for (long it = steps - 1; it >= 0; --it) {
      const cplx<R>* ra = rec + (size_t)it * NR * VEC;
      launch_col_fxa<R, N>(c, B, scheme, S + 1, ra, L.h, s);
      for (int q = S; q >= 1; --q) {
        launch_row_adj<R, N>(c, B, phys_of(it * S + q - 1), s);
        launch_col_fxa<R, N>(c, B, scheme, q, ra, L.h, s);
      }
    }
    return cuda_err(c, cudaGetLastError(), "vjp (RK4 / Lawson-RK6)");
  }

  static int linearize(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                       R* out_fields, ecs_info* info, cudaStream_t s) {
    auto& L = c->lin;
    const bool rk43 = cfg->mode == ECS_MODE_LAWSON_RK43;
    if (cfg->mode == ECS_MODE_TDRK4) return linearize_td(c, cfg, fields, T, sx, out_fields, info, s);
    if (fxl_mode(cfg->mode)) return linearize_fxl(c, cfg, fields, T, sx, out_fields, info, s);
    if (cfg->mode != ECS_MODE_LAWSON_RK4 && !rk43)
      return set_err(c, ECS_ERR_BAD_MODE, "unknown mode");
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    int st = lin_prologue(c, cfg, fields, T, sx, s);
    if (st) return st;
    cudaError_t e = cudaSuccess;
    if (!rk43) {
      const long steps = (long)cfg->num_checkpoints * cfg->ministeps;
      if (steps <= 0) return set_err(c, ECS_ERR_INVALID, "steps must be > 0");
      const long kseg = (cfg->ckpt_every > 0 && cfg->ckpt_every < steps) ? cfg->ckpt_every : 0;
      st = grow(c, &L.rec, &L.rec_bytes, (size_t)(kseg ? kseg : steps) * Q_NREC * vb);
      if (st) return st;
      cudaMemcpyAsync(c->F, L.f0box, vb, cudaMemcpyDeviceToDevice, s);
      st = rk4_setup(c, T, cfg->num_checkpoints, cfg->ministeps, 1, s);
      if (st) return st;
      if (kseg) {   // keep only the segment start states; segments are recomputed by jvp / vjp
        const long nseg = (steps + kseg - 1) / kseg;
        st = grow(c, &L.ckpt, &L.ckpt_bytes, (size_t)nseg * vb);
        if (st) return st;
        for (long g = 0; g < nseg; ++g) {
          cudaMemcpyAsync((cplx<R>*)L.ckpt + (size_t)g * VEC, c->F, vb, cudaMemcpyDeviceToDevice, s);
          st = integrate_rk4(c, 1, std::min(kseg, steps - g * kseg), s);
          if (st) return st;
        }
      } else {
        record_rk4_segment(c, (cplx<R>*)L.rec, steps, s);
      }
      L.seg = kseg;
      L.nrec = steps;
      L.h = (double)(R)((L.T / (double)cfg->num_checkpoints) / (double)cfg->ministeps);
      cudaMemcpyAsync(L.phi, c->F, vb, cudaMemcpyDeviceToDevice, s);
      if (info) { info->completed = 1; info->s = 1.0; info->accepted = (int)steps; info->rejected = 0; info->fevals = (int)(4 * steps); }
    } else {
      const long cap = (long)cfg->checkpoints * cfg->max_steps_per_checkpoint;
      st = lin43_alloc(c, cfg, s);
      if (st) return st;
      st = rk43_solve(c, cfg, T, 1, s, (cplx<R>*)L.rec, L.rec_h, L.rec_acc, (int)cap);
      if (st) return st;
      cudaMemcpyAsync(L.phi, c->F, vb, cudaMemcpyDeviceToDevice, s);
      StepCtl hc;
      e = cudaMemcpyAsync(&hc, c->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return cuda_err(c, e, "linearize readback");
      L.nrec = hc.attempts;
      L.acc.assign(L.nrec, 0); L.hs.assign(L.nrec, 0.0);
      if (L.nrec > 0) {
        e = cudaMemcpyAsync(L.acc.data(), L.rec_acc, L.nrec * sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(L.hs.data(), L.rec_h, L.nrec * sizeof(double), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_err(c, e, "linearize record readback");
      }
      if (info) { info->completed = hc.done; info->s = hc.s; info->accepted = hc.accepted; info->rejected = hc.rejected; info->fevals = hc.fevals; }
    }
    if (out_fields) {
      st = residual(c, cfg, fields, (const cplx<R>*)L.phi, (const cplx<R>*)L.f0box, L.dsx, 1, out_fields, s, 1);
      if (st) return st;
    }
    L.valid = 1;
    return cuda_err(c, cudaGetLastError(), "linearize");
  }

  // out = base - irfft2(sym(Phi)) [- P_sym(base - irfft2(box(base))) in Lawson-RK4(3) mode]
  static int residual(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* base, const cplx<R>* phi, const cplx<R>* basebox,
                      const double* sx, int B, R* out, cudaStream_t s, int sx_shared) {
    const bool rk43 = carry_mode(cfg->mode);   // modes outside the box carried unchanged
    if (rk43) {
      launch_col_from_box<R, N>(c, basebox, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
      launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, (R*)c->fields_tmp2, base, nullptr, B, 1, s);
    }
    launch_col_from_box<R, N>(c, phi, (cplx<R>*)c->G, B, sx, cfg->shift_reflect_ny, cfg->rot, 1, 0, s, sx_shared);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, out, base, nullptr, B, 1, s);
    if (rk43) {
      const int odd = (cfg->shift_reflect_ny % 2 + 2) % 2 == 1;
      ++c->launches; k_sub_sym_phys<R><<<grid1d((long)B * 2 * N * N), 256, 0, s>>>(out, (const R*)c->fields_tmp2, odd, cfg->rot, N, B);
    }
    return cuda_err(c, cudaGetLastError(), "residual");
  }

  // Regeneration plan for the primal physical fields (offsets in box vectors).
  static int upload_items(ecs_ctx* c, const std::vector<long>& items, cudaStream_t s) {
    if (items.size() > c->items_cap) {
      if (c->items) cudaFree(c->items);
      if (cudaMalloc(&c->items, items.size() * sizeof(long)) != cudaSuccess) { c->items = nullptr; c->items_cap = 0; return set_err(c, ECS_ERR_OOM, "items"); }
      c->items_cap = items.size();
    }
    // pageable source: the call returns once the vector has been staged
    return cuda_err(c, cudaMemcpyAsync(c->items, items.data(), items.size() * sizeof(long), cudaMemcpyHostToDevice, s),
                    "items upload");
  }

  // Stage inputs regenerated per chunk (about 384 MiB of buffers; ECS_REGEN_ITEMS overrides).
  static size_t chunk_items(const ecs_ctx* ctx) {
    if (ctx->regen_items > 0) return (size_t)ctx->regen_items;
    const size_t per = (size_t)NG * K * N * sizeof(cplx<R>) + (size_t)N * NPH * N * sizeof(R);
    size_t c = ((size_t)384 << 20) / per;
    return c < 8 ? 8 : (c > 512 ? 512 : c);
  }

  static int ensure_regen(ecs_ctx* c) {
    const size_t ci = chunk_items(c);
    if (c->reg_items >= ci && c->Greg) return ECS_OK;
    size_t have1 = c->Greg ? 1 : 0, have2 = have1;
    (void)have2;
    if (c->Greg) { cudaFree(c->Greg); cudaFree(c->Phys); c->Greg = c->Phys = nullptr; }
    size_t h1 = 0, h2 = 0;
    int st = grow(c, &c->Greg, &h1, ci * NG * K * N * sizeof(cplx<R>));
    if (!st) st = grow(c, &c->Phys, &h2, ci * N * NPH * N * sizeof(R));
    if (st) return st;
    (void)have1;
    c->reg_items = ci;
    return ECS_OK;
  }

  // ---------------------------------------------------------------------
  // JVP of objective_RPO at the current linearisation for B tangents.
  // ---------------------------------------------------------------------
  static int jvp(ecs_ctx* c, const R* dfields, const double* dT, const double* dsx, R* out, double* odT, double* odsx,
                 int B, cudaStream_t s) {
    auto& L = c->lin;
    if (!L.valid) return set_err(c, ECS_ERR_INVALID, "no linearisation: call ecs_linearize first");
    if (L.mode == ECS_MODE_TDRK4) return jvp_td(c, dfields, dT, dsx, out, odT, odsx, B, s);
    if (fxl_mode(L.mode)) return jvp_fxl(c, dfields, dT, dsx, out, odT, odsx, B, s);
    const bool rk43 = L.mode == ECS_MODE_LAWSON_RK43;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const int nslot = rk43 ? (int)S_NSLOT : (int)D_NS4;
    int st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = ensure_regen(c);
    if (st) return st;
    // tangent initial state: box(dfields) into slot X0 (RK4(3)) or F (RK4)
    launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->D + (size_t)(rk43 ? (int)S_X0 : (int)D_F) * VEC, B, 2, s,
                            (long)nslot * VEC);
    // regeneration plan
    std::vector<long> items;
    std::vector<long> item_of;   // first item index per step / attempt (-1 if none)
    if (!rk43) {
      for (long a = 0; a < L.nrec; ++a) {
        item_of.push_back((long)items.size());
        const long base = a * Q_NREC;
        items.push_back(base + Q_F); items.push_back(base + Q_X2); items.push_back(base + Q_X3); items.push_back(base + Q_X4);
      }
    } else {
      items.push_back(RR_X0);   // x0 of attempt 0 (initial k1)
      for (long a = 0; a < L.nrec; ++a) {
        if (!L.acc[a]) { item_of.push_back(-1); continue; }
        item_of.push_back((long)items.size());
        const long base = a * RR_NREC;
        items.push_back(base + RR_Y2); items.push_back(base + RR_Y3); items.push_back(base + RR_Y4); items.push_back(base + RR_XF);
      }
    }
    st = upload_items(c, items, s);
    if (st) return st;
    const long ci = (long)chunk_items(c);
    long chunk_lo = -1;
    auto phys_of = [&](long item) -> const R* {
      if (chunk_lo < 0 || item < chunk_lo || item >= chunk_lo + ci) {
        chunk_lo = item;
        const long cnt = std::min<long>(ci, (long)items.size() - item);
        launch_regen<R, N>(c, (const cplx<R>*)L.rec, c->items + item, (int)cnt, s);
      }
      return (const R*)c->Phys + (size_t)(item - chunk_lo) * N * NPH * N;
    };
    const cplx<R>* rec = (const cplx<R>*)L.rec;
    if (!rk43) {
      const double dscale = 1.0 / ((double)L.cfg.num_checkpoints * (double)L.cfg.ministeps);
      const long kseg = L.seg ? L.seg : L.nrec;
      for (long a0 = 0; a0 < L.nrec; a0 += kseg) {
        const long cnt = std::min(kseg, L.nrec - a0);
        const cplx<R>* rseg = rk4_segment_record(c, a0, cnt, s);
        std::vector<long> sitems;
        for (long it = 0; it < cnt; ++it) {
          const long base = it * Q_NREC;
          sitems.push_back(base + Q_F); sitems.push_back(base + Q_X2); sitems.push_back(base + Q_X3); sitems.push_back(base + Q_X4);
        }
        st = upload_items(c, sitems, s);
        if (st) return st;
        long slo = -1;
        auto sphys = [&](long item) -> const R* {
          if (slo < 0 || item < slo || item >= slo + ci) {
            slo = item;
            launch_regen<R, N>(c, rseg, c->items + item, (int)std::min<long>(ci, (long)sitems.size() - item), s);
          }
          return (const R*)c->Phys + (size_t)(item - slo) * N * NPH * N;
        };
        launch_col_tan<R, N>(c, B, TS_START, 1, rseg, dT, 0.0, L.h, dscale, nslot, s);
        for (long it = 0; it < cnt; ++it) {
          const cplx<R>* ra = rseg + (size_t)it * Q_NREC * VEC;
          for (int k = 1; k <= 4; ++k) {
            launch_row_tan<R, N>(c, B, sphys(4 * it + (k - 1)), s);
            launch_col_tan<R, N>(c, B, k, (k == 4 && it == cnt - 1) ? 0 : 1, ra, dT, 0.0, L.h, dscale, nslot, s);
          }
        }
      }
    } else {
      const std::vector<ChainOp> ops = rk43_tangent_ops(L, item_of);
      if (use_chain(c, B)) {
        st = run_chain(c, ops, ci, (long)items.size(), B, nslot, dT, s);
        if (st) return st;
      } else {
        for (const ChainOp& op : ops) {
          const cplx<R>* ra = rec + (size_t)op.rec * VEC;
          if (op.kind == CH_ROW) {
            launch_row_tan<R, N>(c, B, phys_of(op.item), s);
          } else if (op.kind == CH_REJECT) {
            ++c->launches; k_tan_reject<R><<<grid1d((long)B * VEC), 256, 0, s>>>((cplx<R>*)c->D, nslot, ra, dT, 1.0, N, B);
          } else {
            launch_col_tan<R, N>(c, B, op.stage, op.produce, ra, dT, L.T, op.h, 1.0, nslot, s, nullptr, 0, nullptr,
                                 nullptr, op.stage == T43_EA ? rec + (size_t)op.rec2 * VEC : nullptr);
          }
        }
      }
    }
    return jvp_finish(c, dfields, dsx, out, odT, odsx, B, s);
  }

  // The passes of the adaptive tangent sweep in launch order: inverse transforms
  // of dX0, the row pass at x0 and the initial dk1, then per accepted attempt
  // the stages A..E with a row pass before B..E (E of an attempt followed by an
  // accepted attempt runs that attempt's A too: T43_EA), per rejected attempt
  // the update of the carried dk1.  Row-pass items index the regeneration plan
  // (item_of: first item of each accepted attempt; item 0 is x0 of attempt 0).
  static std::vector<ChainOp> rk43_tangent_ops(const ecs_ctx::Lin& L, const std::vector<long>& item_of) {
    std::vector<ChainOp> ops;
    ops.reserve((size_t)L.nrec * 8 + 4);
    auto col = [&](int stage, int produce, long a, double h, long a2 = 0) {
      ChainOp o{}; o.kind = CH_COL; o.stage = stage; o.produce = produce;
      o.rec = a * RR_NREC; o.rec2 = a2 * RR_NREC; o.h = h; ops.push_back(o);
    };
    auto row = [&](long item) { ChainOp o{}; o.kind = CH_ROW; o.item = item; ops.push_back(o); };
    col(T43_START, 1, 0, 0.0);
    row(0);
    col(T43_INIT, 0, 0, 0.0);
    bool a_started = false;   // the E pass of the previous attempt ran this one's A pass (T43_EA)
    for (long a = 0; a < L.nrec; ++a) {
      const double h = L.hs[a];
      if (!L.acc[a]) {
        ChainOp o{}; o.kind = CH_REJECT; o.rec = a * RR_NREC; ops.push_back(o);
        a_started = false;
        continue;
      }
      if (!a_started) col(T43_A, 1, a, h);
      const bool merge = a + 1 < L.nrec && L.acc[a + 1];
      for (int k = 0; k < 4; ++k) {
        row(item_of[a] + k);
        if (k == 3 && merge) col(T43_EA, 1, a, L.hs[a + 1], a + 1);
        else col(T43_B + k, 1, a, h);
      }
      a_started = merge;
    }
    return ops;
  }

  // Batches that the adaptive tangent sweep runs through the cluster-resident
  // pass list (k_tan_chain): see chain_batch.
  static bool use_chain(const ecs_ctx* c, int B) { return chain_batch(c, B, c->chain_minb, c->chain_maxb); }

  // The pass list through k_tan_chain: one launch per regeneration chunk (the
  // row passes of a launch read the chunk's physical fields), with the chunk's
  // regeneration launched before it on the same stream.
  static int run_chain(ecs_ctx* c, const std::vector<ChainOp>& ops, long ci, long nitems, int B, int nslot,
                       const double* dT, cudaStream_t s) {
    if constexpr (N <= 128) {
      auto& L = c->lin;
      int st = grow(c, &c->chain_ops, &c->chain_ops_bytes, ops.size() * sizeof(ChainOp));
      if (st) return st;
      st = cuda_err(c, cudaMemcpyAsync(c->chain_ops, ops.data(), ops.size() * sizeof(ChainOp), cudaMemcpyHostToDevice, s),
                    "pass list upload");
      if (st) return st;
      ChainParams<R> P{};
      ColTanParams<R>& cp = P.col;
      cp.H = (const cplx<R>*)c->H; cp.G = (cplx<R>*)c->G; cp.D = (cplx<R>*)c->D; cp.nslot = nslot;
      cp.dT = dT; cp.t = L.T; cp.dscale = 1.0; cp.tw = (const cplx<R>*)c->tw; cp.nu = (R)c->nu; cp.eta = (R)c->eta;
      cp.B = B;
      P.row.G = (const cplx<R>*)c->G; P.row.H = (cplx<R>*)c->H; P.row.tw = (const cplx<R>*)c->tw; P.row.B = B;
      P.rec = (const cplx<R>*)L.rec;
      P.ops = (const ChainOp*)c->chain_ops;
      long chunk_lo = -1;
      size_t start = 0;
      auto flush = [&](size_t end) {
        if (end <= start) return;
        P.op0 = (int)start; P.op1 = (int)end;
        P.phys = (const R*)c->Phys; P.item0 = chunk_lo < 0 ? 0 : chunk_lo;
        const bool dsh = c->chain_dsh != 0;
        auto go = [&](auto w, auto dsm) {
          constexpr int W = decltype(w)::value;
          constexpr bool DSM = decltype(dsm)::value;
          if (W == 8 && dsh)
            launch_cluster(c, B, chain_cl<N, W>(), k_tan_chain<R, N, W, DSM, W == 8>, dim3(B * chain_cl<N, W>()),
                           dim3(W * 32), chain_smem<R, N, W, DSM, W == 8>(), s, P);
          else
            launch_cluster(c, B, chain_cl<N, W>(), k_tan_chain<R, N, W, DSM, false>, dim3(B * chain_cl<N, W>()),
                           dim3(W * 32), chain_smem<R, N, W, DSM, false>(), s, P);
        };
        chain_dispatch(c, B, false, go);
        start = end;
      };
      for (size_t i = 0; i < ops.size(); ++i) {
        if (ops[i].kind != CH_ROW) continue;
        const long item = ops[i].item;
        if (chunk_lo < 0 || item < chunk_lo || item >= chunk_lo + ci) {
          if (chunk_lo >= 0) flush(i);   // the passes before the first row pass read no physical fields
          chunk_lo = item;
          const long cnt = std::min<long>(ci, nitems - item);
          launch_regen<R, N>(c, (const cplx<R>*)L.rec, c->items + item, (int)cnt, s);
        }
      }
      flush(ops.size());
      return cuda_err(c, cudaGetLastError(), "tangent pass list");
    } else {
      (void)ops; (void)ci; (void)nitems; (void)B; (void)nslot; (void)dT; (void)s;
      return set_err(c, ECS_ERR_UNSUPPORTED, "pass list: n > 128");
    }
  }

  // JVP output from the final tangent state:
  // d fields = dfields - irfft2(sym(dPhi + i kx dsx Phi)) [- rest term]; phase-condition tangents.
  static int jvp_finish(ecs_ctx* c, const R* dfields, const double* dsx, R* out, double* odT, double* odsx, int B,
                        cudaStream_t s) {
    auto& L = c->lin;
    const bool rk43 = L.mode == ECS_MODE_LAWSON_RK43, td = L.mode == ECS_MODE_TDRK4, fxl = fxl_mode(L.mode);
    const size_t VEC = 2UL * K * M;
    const int nslot = rk43 ? (int)S_NSLOT : td ? (int)DT_NSLOT : fxl ? fxt_nslot(fx_scheme(L.mode)) : (int)D_NS4;
    const int fslot = rk43 ? (int)S_X0 : td ? (int)DT_F : fxl ? (int)FT_F : (int)D_F;
    ++c->launches; k_tan_shift<R><<<grid1d((long)B * VEC), 256, 0, s>>>((const cplx<R>*)c->D + (size_t)fslot * VEC,
                                                         (long)nslot * VEC, (const cplx<R>*)L.phi, dsx,
                                                         (cplx<R>*)c->V, N, B);
    if (carry_mode(L.mode)) {   // box(dfields) for the rest term
      launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
      launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->OUT, B, 2, s);
    }
    int st = residual(c, &L.cfg, dfields, (const cplx<R>*)c->V, (const cplx<R>*)c->OUT, L.dsx, B, out, s, 1);
    if (st) return st;
    ++c->launches; k_phase_dot<R><<<B, 256, 0, s>>>((const R*)L.vt, (const R*)L.vx, dfields, odT, odsx, N);
    return cuda_err(c, cudaGetLastError(), "jvp");
  }

  // Streams, events and buffers of the pipelined linearisation (allocations
  // synchronise the device, so they all happen before the pipelined phase).
  static int ensure_pipeline(ecs_ctx* c, long amax) {
    constexpr int GA = 16;
    if (!c->pstream) {
      int lo = 0, hi = 0;
      cudaError_t e = cudaDeviceGetStreamPriorityRange(&lo, &hi);
      if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&c->pstream, cudaStreamNonBlocking, hi);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->pev[0], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->pev[1], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->tfork, cudaEventDisableTiming);
      for (int g = 0; g < ecs_ctx::MAXG && e == cudaSuccess; ++g) {   // group 0 runs on the caller's stream
        if (g > 0) e = cudaStreamCreateWithFlags(&c->tstream[g], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->tjoin[g][0], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->tjoin[g][1], cudaEventDisableTiming);
      }
      if (e == cudaSuccess) e = cudaMalloc(&c->Gp, (size_t)NG * K * N * sizeof(cplx<R>));
      if (e == cudaSuccess) e = cudaMalloc(&c->Hp, (size_t)NHA * K * N * sizeof(cplx<R>));
      if (e == cudaSuccess) e = cudaHostAlloc((void**)&c->hctl, 2 * sizeof(StepCtl), cudaHostAllocDefault);
      if (e == cudaSuccess) e = cudaHostAlloc((void**)&c->hchunk_acc, 2 * GA * sizeof(int), cudaHostAllocDefault);
      if (e == cudaSuccess) e = cudaHostAlloc((void**)&c->hchunk_h, 2 * GA * sizeof(double), cudaHostAllocDefault);
      if (e != cudaSuccess) return cuda_err(c, e, "pipeline set-up");
    }
    const size_t need = (size_t)(4 * amax + 1);
    if (c->hitems_cap < need) {
      if (c->hitems) cudaFreeHost(c->hitems);
      c->hitems = nullptr; c->hitems_cap = 0;
      if (cudaHostAlloc((void**)&c->hitems, need * sizeof(long), cudaHostAllocDefault) != cudaSuccess)
        return set_err(c, ECS_ERR_OOM, "item staging");
      c->hitems_cap = need;
    }
    if (c->items_cap < need) {
      if (c->items) cudaFree(c->items);
      c->items = nullptr; c->items_cap = 0;
      if (cudaMalloc(&c->items, need * sizeof(long)) != cudaSuccess) return set_err(c, ECS_ERR_OOM, "items");
      c->items_cap = need;
    }
    return ECS_OK;
  }

  // Fixed-step Lawson-RK4 form of linearize_jvp (full record): the batch-1
  // primal records chunks of steps on the primal stream, each followed by an
  // event; the tangent sweep of a chunk (regeneration of its primal fields
  // included) waits on that event on the caller's stream.  No host round trip:
  // the host queues both streams ahead.
  static int linearize_jvp_rk4(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T,
                               const double* sx, R* out_fields, ecs_info* info, const R* dfields, const double* dT,
                               const double* dsx, R* out, double* odT, double* odsx, int B, cudaStream_t s) {
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const long steps = (long)cfg->num_checkpoints * cfg->ministeps;
    const int nslot = (int)D_NS4;
    int st = ensure_pipeline(c, steps);
    if (!st) st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = ensure_regen(c);
    if (!st) st = lin_prologue(c, cfg, fields, T, sx, s);
    if (!st) st = grow(c, &L.rec, &L.rec_bytes, (size_t)steps * Q_NREC * vb);
    if (st) return st;
    cudaMemcpyAsync(c->F, L.f0box, vb, cudaMemcpyDeviceToDevice, s);
    st = rk4_setup(c, T, cfg->num_checkpoints, cfg->ministeps, 1, s);
    if (st) return st;
    L.seg = 0;
    L.nrec = steps;
    L.h = (double)(R)((L.T / (double)cfg->num_checkpoints) / (double)cfg->ministeps);
    L.acc.clear(); L.hs.clear();
    const double dscale = 1.0 / ((double)cfg->num_checkpoints * (double)cfg->ministeps);
    // tangent initial state: box(dfields) into slot F; regeneration items (4 per step) staged once
    launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->D + (size_t)D_F * VEC, B, 2, s, (long)nslot * VEC);
    for (long it = 0; it < steps; ++it) {
      long* q = c->hitems + 4 * it;
      const long base = it * Q_NREC;
      q[0] = base + Q_F; q[1] = base + Q_X2; q[2] = base + Q_X3; q[3] = base + Q_X4;
    }
    cudaError_t e = cudaMemcpyAsync(c->items, c->hitems, 4 * steps * sizeof(long), cudaMemcpyHostToDevice, s);
    cudaStream_t ps = c->pstream;
    if (e == cudaSuccess) e = cudaEventRecord(c->pev[0], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ps, c->pev[0], 0);
    if (e != cudaSuccess) return cuda_err(c, e, "pipeline fork");
    cplx<R>* rec = (cplx<R>*)L.rec;
    const long ci = (long)chunk_items(c);
    const long CS = std::max(1L, std::min(16L, ci / 4));   // steps per chunk (their items fit one regeneration)
    const long nch = (steps + CS - 1) / CS;
    auto primal_chunk = [&](long k) -> cudaError_t {
      void* const Gs = c->G; void* const Hs = c->H;
      c->G = c->Gp; c->H = c->Hp;
      PlainOrder plain_order(c);
      if (k == 0) launch_col_rk4<R, N>(c, 1, COL_START, 1, 0, ps);
      for (long it = k * CS; it < std::min(steps, (k + 1) * CS); ++it) {
        cplx<R>* rs = rec + (size_t)it * Q_NREC * VEC;
        for (int q = 1; q <= 4; ++q) {
          launch_row_rhs<R, N>(c, 1, ps);
          launch_col_rk4<R, N>(c, 1, q, (q == 4 && it == steps - 1) ? 0 : 1, 0, ps, rs, 0);
        }
      }
      c->G = Gs; c->H = Hs;
      return cudaEventRecord(c->pev[k & 1], ps);
    };
    auto tangent_chunk = [&](long k) -> cudaError_t {
      cudaError_t e2 = cudaStreamWaitEvent(s, c->pev[k & 1], 0);
      if (e2 != cudaSuccess) return e2;
      const long a0 = k * CS, cnt = std::min(steps, (k + 1) * CS) - a0;
      launch_regen<R, N>(c, rec, c->items + 4 * a0, (int)(4 * cnt), s);
      if (k == 0) launch_col_tan<R, N>(c, B, TS_START, 1, rec, dT, 0.0, L.h, dscale, nslot, s);
      for (long it = a0; it < a0 + cnt; ++it) {
        const cplx<R>* ra = rec + (size_t)it * Q_NREC * VEC;
        for (int q = 1; q <= 4; ++q) {
          launch_row_tan<R, N>(c, B, (const R*)c->Phys + (size_t)(4 * (it - a0) + q - 1) * N * NPH * N, s);
          launch_col_tan<R, N>(c, B, q, (q == 4 && it == steps - 1) ? 0 : 1, ra, dT, 0.0, L.h, dscale, nslot, s);
        }
      }
      return cudaGetLastError();
    };
    // chunk k+1 of the primal is queued before the tangents of chunk k (each event is
    // waited on before the chunk two ahead records it again)
    e = primal_chunk(0);
    for (long k = 0; k < nch && e == cudaSuccess; ++k) {
      if (k + 1 < nch) e = primal_chunk(k + 1);
      if (e == cudaSuccess) e = tangent_chunk(k);
    }
    if (e != cudaSuccess) return cuda_err(c, e, "pipelined linearisation");
    cudaMemcpyAsync(L.phi, c->F, vb, cudaMemcpyDeviceToDevice, s);
    if (info) { info->completed = 1; info->s = 1.0; info->accepted = (int)steps; info->rejected = 0; info->fevals = (int)(4 * steps); }
    if (out_fields) {
      st = residual(c, cfg, fields, (const cplx<R>*)L.phi, (const cplx<R>*)L.f0box, L.dsx, 1, out_fields, s, 1);
      if (st) return st;
    }
    L.valid = 1;
    return jvp_finish(c, dfields, dsx, out, odT, odsx, B, s);
  }

  // ---------------------------------------------------------------------
  // Linearisation and JVP in one call, pipelined (Lawson-RK4(3)), as jax.jvp
  // returns (objective, J v) together.  The batch-1 primal solve runs on a
  // high-priority context stream with its own scratch, in chunks of GA
  // attempts (the captured attempt graph); after each chunk the host reads back
  // the control block and accept flags and queues the tangent sweep over those
  // attempts on the caller's stream behind the chunk's event.  The primal
  // occupies a few SMs, the tangent batch the rest, so the primal is hidden
  // behind the tangents.  Every kernel sees the same inputs as in
  // ecs_linearize followed by ecs_jvp, so the results are the same.  Fixed-step
  // mode, or an attempt cap that is not a multiple of GA, runs the two in sequence.
  // ---------------------------------------------------------------------
  static int linearize_jvp(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                           R* out_fields, ecs_info* info, const R* dfields, const double* dT, const double* dsx,
                           R* out, double* odT, double* odsx, int B, cudaStream_t s) {
    constexpr int GA = 16;
    const long amax = (long)cfg->checkpoints * cfg->max_steps_per_checkpoint;
    const long steps4 = (long)cfg->num_checkpoints * cfg->ministeps;
    if (cfg->mode == ECS_MODE_LAWSON_RK4 && steps4 > 0 && !(cfg->ckpt_every > 0 && cfg->ckpt_every < steps4))
      return linearize_jvp_rk4(c, cfg, fields, T, sx, out_fields, info, dfields, dT, dsx, out, odT, odsx, B, s);
    if (cfg->mode != ECS_MODE_LAWSON_RK43 || amax < GA || amax % GA != 0) {
      const int st = linearize(c, cfg, fields, T, sx, out_fields, info, s);
      return st ? st : jvp(c, dfields, dT, dsx, out, odT, odsx, B, s);
    }
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const int nslot = (int)S_NSLOT;
    int st = ensure_pipeline(c, amax);
    if (!st) st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = ensure_regen(c);
    if (!st) st = lin_prologue(c, cfg, fields, T, sx, s);
    if (!st) st = lin43_alloc(c, cfg, s);
    if (st) return st;
    const cplx<R>* rec = (const cplx<R>*)L.rec;
    // tangent initial state: box(dfields) into slot X0
    launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->D + (size_t)S_X0 * VEC, B, 2, s, (long)nslot * VEC);
    // primal set-up and attempt graph on the primal stream, after everything queued so far
    cudaStream_t ps = c->pstream;
    cudaError_t e = cudaEventRecord(c->pev[0], s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(ps, c->pev[0], 0);
    if (e != cudaSuccess) return cuda_err(c, e, "pipeline fork");
    void* const Gs = c->G; void* const Hs = c->H;
    c->G = c->Gp; c->H = c->Hp;
    st = rk43_solve(c, cfg, T, 1, ps, (cplx<R>*)L.rec, L.rec_h, L.rec_acc, (int)amax, false);
    c->G = Gs; c->H = Hs;
    if (st) return st;
    const auto& gk = c->g43;
    auto launch_chunk = [&](long chunk, int bi) -> cudaError_t {
      cudaError_t e2 = cudaGraphLaunch(gk.exec, ps);
      c->launches += gk.nodes;
      if (e2 == cudaSuccess) e2 = cudaMemcpyAsync(c->hctl + bi, c->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, ps);
      if (e2 == cudaSuccess)
        e2 = cudaMemcpyAsync(c->hchunk_acc + bi * GA, L.rec_acc + chunk * GA, GA * sizeof(int), cudaMemcpyDeviceToHost, ps);
      if (e2 == cudaSuccess)
        e2 = cudaMemcpyAsync(c->hchunk_h + bi * GA, L.rec_h + chunk * GA, GA * sizeof(double), cudaMemcpyDeviceToHost, ps);
      if (e2 == cudaSuccess) e2 = cudaEventRecord(c->pev[bi], ps);
      return e2;
    };
    // Tangent sweep over attempts [a_lo, a_hi) whose record is complete.  The
    // batch is split into groups (of at least 16 tangents) swept on their own
    // streams (group 0 on the caller's stream), so that one group's row kernels
    // and another's column kernels share the SMs and fill each other's tails.
    // The attempts' primal fields are regenerated per chunk on the caller's
    // stream, into alternating halves of the regeneration buffer when two
    // chunks fit.
    L.acc.clear(); L.hs.clear();
    const long ci = (long)chunk_items(c);
    const int ngrp = std::max(1, std::min(c->tgroups, B / 16));
    int bsplit[ecs_ctx::MAXG + 1];
    for (int g = 0; g <= ngrp; ++g) bsplit[g] = (int)((long)B * g / ngrp);
    const bool dbl = ci >= 2 * (4 * GA + 1);
    bool joined[ecs_ctx::MAXG][2];
    for (auto& j : joined) j[0] = j[1] = true;
    long nitems = 0;
    int half = 0;
    const double t = L.T;
    std::vector<long> item_of;
    auto sweep = [&](int g, long a_lo, long a_hi, const int* acc, const double* hh, const R* phys0, long item_lo) {
      const int b0 = bsplit[g], Bg = bsplit[g + 1] - b0;
      cudaStream_t st = g == 0 ? s : c->tstream[g];
      void* const G0 = c->G; void* const H0 = c->H; void* const D0 = c->D;
      c->G = (cplx<R>*)G0 + (size_t)b0 * NG * K * N;
      c->H = (cplx<R>*)H0 + (size_t)b0 * NH * K * N;
      c->D = (cplx<R>*)D0 + (size_t)b0 * nslot * VEC;
      const double* dTg = dT + b0;
      auto phys = [&](long item) { return phys0 + (size_t)(item - item_lo) * N * NPH * N; };
      if (a_lo == 0) {
        launch_col_tan<R, N>(c, Bg, T43_START, 1, rec, dTg, t, 0.0, 1.0, nslot, st);
        launch_row_tan<R, N>(c, Bg, phys(0), st);
        launch_col_tan<R, N>(c, Bg, T43_INIT, 0, rec, dTg, t, 0.0, 1.0, nslot, st);
      }
      // The E column pass of an accepted attempt and the A column pass of the
      // next one, when that one is accepted and in this chunk, run as one
      // launch (T43_EA: the same arithmetic, in registers instead of slots).
      bool a_started = false;
      for (long a = a_lo; a < a_hi; ++a) {
        const cplx<R>* ra = rec + (size_t)a * RR_NREC * VEC;
        const double h = hh[a - a_lo];
        if (!acc[a - a_lo]) {
          ++c->launches; k_tan_reject<R><<<grid1d((long)Bg * VEC), 256, 0, st>>>((cplx<R>*)c->D, nslot, ra, dTg, 1.0, N, Bg);
          a_started = false;
          continue;
        }
        const bool kt = g == 0 && c->kt.on;
        if (!a_started) {
          if (kt) kt_begin(c, st);
          launch_col_tan<R, N>(c, Bg, T43_A, 1, ra, dTg, t, h, 1.0, nslot, st);
          if (kt) kt_end(c, 1, Bg, st);
        }
        const bool merge = a + 1 < a_hi && acc[a + 1 - a_lo];
        for (int k = 0; k < 4; ++k) {
          if (kt) kt_begin(c, st);
          launch_row_tan<R, N>(c, Bg, phys(item_of[a - a_lo] + k), st);
          if (kt) { kt_end(c, 0, Bg, st); kt_begin(c, st); }
          if (k == 3 && merge)
            launch_col_tan<R, N>(c, Bg, T43_EA, 1, ra, dTg, t, hh[a + 1 - a_lo], 1.0, nslot, st, nullptr, 0, nullptr,
                                 nullptr, ra + (size_t)RR_NREC * VEC);
          else
            launch_col_tan<R, N>(c, Bg, T43_B + k, 1, ra, dTg, t, h, 1.0, nslot, st);
          if (kt) kt_end(c, 1, Bg, st);
        }
        a_started = merge;
      }
      c->G = G0; c->H = H0; c->D = D0;
    };
    auto tangent_chunk = [&](long a_lo, long a_hi, const int* acc, const double* hh) -> int {
      const long i0 = nitems;
      long* stage = c->hitems + i0;
      long cnt = 0;
      if (a_lo == 0) stage[cnt++] = RR_X0;   // x0 of attempt 0 (initial k1)
      item_of.assign(a_hi - a_lo, -1);
      for (long a = a_lo; a < a_hi; ++a) {
        L.acc.push_back(acc[a - a_lo]); L.hs.push_back(hh[a - a_lo]);
        if (!acc[a - a_lo]) continue;
        item_of[a - a_lo] = i0 + cnt;
        const long base = a * RR_NREC;
        stage[cnt++] = base + RR_Y2; stage[cnt++] = base + RR_Y3; stage[cnt++] = base + RR_Y4; stage[cnt++] = base + RR_XF;
      }
      nitems += cnt;
      cudaError_t e2 = cudaSuccess;
      const int hb = dbl ? half : 0;
      R* phys0 = (R*)c->Phys + (dbl ? (size_t)hb * (ci / 2) * N * NPH * N : 0);
      if (cnt > 0) {
        e2 = cudaMemcpyAsync(c->items + i0, stage, cnt * sizeof(long), cudaMemcpyHostToDevice, s);
        // the other groups' last reads of this half must be done before it is overwritten
        for (int g = 1; g < ngrp && e2 == cudaSuccess; ++g)
          if (!joined[g][hb]) { e2 = cudaStreamWaitEvent(s, c->tjoin[g][hb], 0); joined[g][hb] = true; }
        if (e2 != cudaSuccess) return cuda_err(c, e2, "item upload");
        launch_regen<R, N>(c, rec, c->items + i0, (int)cnt, s, phys0);
      }
      if (ngrp > 1) {
        e2 = cudaEventRecord(c->tfork, s);
        if (e2 != cudaSuccess) return cuda_err(c, e2, "tangent fork");
        for (int g = 1; g < ngrp; ++g) {
          e2 = cudaStreamWaitEvent(c->tstream[g], c->tfork, 0);
          if (e2 != cudaSuccess) return cuda_err(c, e2, "tangent fork");
          sweep(g, a_lo, a_hi, acc, hh, phys0, i0);
          e2 = cudaEventRecord(c->tjoin[g][hb], c->tstream[g]);
          if (e2 != cudaSuccess) return cuda_err(c, e2, "tangent join");
          joined[g][hb] = false;
        }
      }
      sweep(0, a_lo, a_hi, acc, hh, phys0, i0);
      if (dbl) half ^= 1;
      return cuda_err(c, cudaGetLastError(), "pipelined tangent");
    };
    // chunk i+1 of the primal is queued before the tangents of chunk i
    long launched = 1, a_done = 0;
    int bi = 0;
    e = launch_chunk(0, 0);
    StepCtl hc{};
    while (true) {
      if (e == cudaSuccess) e = cudaEventSynchronize(c->pev[bi]);
      if (e != cudaSuccess) return cuda_err(c, e, "pipelined linearisation");
      hc = c->hctl[bi];
      const long a_now = hc.attempts;
      const bool more = !hc.done && launched * GA < amax;
      if (more) { e = launch_chunk(launched, bi ^ 1); ++launched; }
      if (e == cudaSuccess) e = cudaStreamWaitEvent(s, c->pev[bi], 0);
      if (e != cudaSuccess) return cuda_err(c, e, "pipelined linearisation");
      st = tangent_chunk(a_done, a_now, c->hchunk_acc + bi * GA, c->hchunk_h + bi * GA);
      if (st) return st;
      a_done = a_now;
      if (!more) break;
      bi ^= 1;
    }
    // join the tangent groups; primal epilogue on the caller's stream (it waited for every chunk)
    for (int g = 1; g < ngrp; ++g)
      for (int hb = 0; hb < 2; ++hb)
        if (!joined[g][hb]) {
          e = cudaStreamWaitEvent(s, c->tjoin[g][hb], 0);
          if (e != cudaSuccess) return cuda_err(c, e, "tangent join");
        }
    ++c->launches; k_rk43_resolve<R><<<grid1d((long)VEC), 256, 0, s>>>((cplx<R>*)c->S43, c->ctl, (cplx<R>*)c->F, N, 1);
    cudaMemcpyAsync(L.phi, c->F, vb, cudaMemcpyDeviceToDevice, s);
    L.nrec = a_done;
    if (info) { info->completed = hc.done; info->s = hc.s; info->accepted = hc.accepted; info->rejected = hc.rejected; info->fevals = hc.fevals; }
    if (out_fields) {
      st = residual(c, cfg, fields, (const cplx<R>*)L.phi, (const cplx<R>*)L.f0box, L.dsx, 1, out_fields, s, 1);
      if (st) return st;
    }
    L.valid = 1;
    return jvp_finish(c, dfields, dsx, out, odT, odsx, B, s);
  }

  // TDRK4 adjoint sweep, last step first (see kernels_fx.cuh); the primal's
  // f, f_temp (with the mean field) and k1, k2 are regenerated per chunk of steps.
  static int vjp_td_sweep(ecs_ctx* c, int B, int nslot, cudaStream_t s) {
    auto& L = c->lin;
    const size_t VEC = 2UL * K * M;
    int st = grow(c, &c->Gx, &c->Gx_bytes, (size_t)B * NHA * K * N * sizeof(cplx<R>));
    if (st) return st;
    const long steps = L.nrec;
    const long ci = (long)chunk_items(c);
    const long CS = std::max(1L, std::min(64L, ci / 4));
    std::vector<long> items;
    items.reserve((size_t)(4 * steps));
    for (long a0 = 0; a0 < steps; a0 += CS) {
      const long cnt = std::min(CS, steps - a0);
      for (long it = a0; it < a0 + cnt; ++it) { items.push_back(it * TR_NREC + TR_F); items.push_back(it * TR_NREC + TR_FT); }
      for (long it = a0; it < a0 + cnt; ++it) { items.push_back(it * TR_NREC + TR_K1); items.push_back(it * TR_NREC + TR_K2); }
    }
    st = upload_items(c, items, s);
    if (st) return st;
    const cplx<R>* rec = (const cplx<R>*)L.rec;
    const size_t pst = (size_t)N * NPH * N;
    const double h = L.h;
    auto col = [&](int stage, const cplx<R>* ra) {
      ColTdaParams<R> p; p.Ha = (const cplx<R>*)c->H; p.Hb = (const cplx<R>*)c->Gx; p.G = (cplx<R>*)c->G;
      p.J = (cplx<R>*)c->D; p.nslot = nslot; p.rec = ra; p.hacc = c->hacc; p.h = h; p.tw = (const cplx<R>*)c->tw;
      p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B;
      const int cols = B * K * 2;
      const dim3 g((cols + COLWARPS - 1) / COLWARPS), bl(COLWARPS * 32);
      switch (stage) {
        case TA_SEED: launch_step(c, B, k_col_tda<R, N, TA_SEED>, g, bl, 0, s, p); break;
        case TA_B: launch_step(c, B, k_col_tda<R, N, TA_B>, g, bl, 0, s, p); break;
        case TA_C: launch_step(c, B, k_col_tda<R, N, TA_C>, g, bl, 0, s, p); break;
        case TA_D: launch_step(c, B, k_col_tda<R, N, TA_D>, g, bl, 0, s, p); break;
        default: launch_step(c, B, k_col_tda<R, N, TA_E>, g, bl, 0, s, p); break;
      }
    };
    auto row2 = [&](const R* pa, const R* pb) {
      RowAdj2Params<R> p; p.G = (const cplx<R>*)c->G; p.Ha = (cplx<R>*)c->H; p.Hb = (cplx<R>*)c->Gx;
      p.phys_a = pa; p.phys_b = pb; p.tw = (const cplx<R>*)c->tw; p.B = B;
      launch_step(c, B, k_row_adj2<R, N, XT>, dim3(B * (N / XT)), dim3(XT * 32), smem_row_rhs<R, N>(), s, p);
    };
    const long nch = (steps + CS - 1) / CS;
    for (long ch = nch - 1; ch >= 0; --ch) {
      const long a0 = ch * CS, cnt = std::min(CS, steps - a0);
      R* P = (R*)c->Phys;
      launch_regen<R, N>(c, rec, c->items + 4 * a0, (int)(2 * cnt), s, P, true);
      launch_regen<R, N>(c, rec, c->items + 4 * a0 + 2 * cnt, (int)(2 * cnt), s, P + 2 * cnt * pst, false);
      for (long it = a0 + cnt - 1; it >= a0; --it) {
        const cplx<R>* ra = rec + (size_t)it * TR_NREC * VEC;
        const R* pf = P + (size_t)(2 * (it - a0)) * pst;
        const R* pft = pf + pst;
        const R* pk1 = P + (size_t)(2 * cnt + 2 * (it - a0)) * pst;
        const R* pk2 = pk1 + pst;
        col(TA_SEED, ra);
        row2(pft, pk2);                      // N'(f_temp)^T, N'(k2)^T of h a2bar
        col(TA_B, ra);
        launch_row_adj<R, N>(c, B, pft, s);  // N'(f_temp)^T of h k2bar
        col(TA_C, ra);
        row2(pf, pk1);                       // N'(f)^T, N'(k1)^T of h a1bar
        col(TA_D, ra);
        launch_row_adj<R, N>(c, B, pf, s);   // N'(f)^T of h k1bar
        col(TA_E, ra);
      }
    }
    return cuda_err(c, cudaGetLastError(), "vjp (TDRK4)");
  }

  // ---------------------------------------------------------------------
  // VJP of objective_RPO at the current linearisation for B cotangents.
  // ---------------------------------------------------------------------
  static int vjp(ecs_ctx* c, const R* cfields, const double* cT, const double* csx, R* gfields, double* gT,
                 double* gsx, int B, cudaStream_t s) {
    auto& L = c->lin;
    if (!L.valid) return set_err(c, ECS_ERR_INVALID, "no linearisation: call ecs_linearize first");
    const bool rk43 = L.mode == ECS_MODE_LAWSON_RK43, td = L.mode == ECS_MODE_TDRK4, fxl = fxl_mode(L.mode);
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>);
    const int nslot = rk43 ? (int)JJ_NS43 : td ? (int)JT_NSLOT : fxl ? fxa_nslot(fx_scheme(L.mode)) : (int)J_NS4;
    const int fslot = rk43 ? (int)JJ_X0 : td ? (int)JT_F : fxl ? (int)FA_F : (int)J_OB;   // cotangent of the final / initial state
    int st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = ensure_regen(c);
    if (!st) st = grow(c, (void**)&c->hacc, &c->hacc_bytes, (size_t)B * K * 2 * sizeof(double));
    if (st) return st;
    cudaMemsetAsync(c->D, 0, (size_t)B * nslot * vb, s);
    cudaMemsetAsync(c->hacc, 0, (size_t)B * K * 2 * sizeof(double), s);
    // head: Ybar = -(c/n^2) rfft2(c_fields) on the box; Phibar = sym^T(Ybar); sxbar
    launch_row_to_box<R, N>(c, cfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->V, B, 2, s);
    ++c->launches; k_box_scale_c<R><<<grid1d((long)B * VEC), 256, 0, s>>>((cplx<R>*)c->V, (long)VEC, N, B, R(-1) / (R(N) * R(N)));
    const int odd = (L.cfg.shift_reflect_ny % 2 + 2) % 2 == 1;
    const double sy = (L.cfg.shift_reflect_ny * 2 * M_PI) / 8;
    ++c->launches; k_adj_head<R><<<B, 256, 0, s>>>((const cplx<R>*)c->V, (const cplx<R>*)L.phi, L.dsx, 1, sy, odd, L.cfg.rot,
                                     (cplx<R>*)c->D + (size_t)fslot * VEC, (long)nslot * VEC,
                                     gsx, N);
    double tscale = 1.0;
    if (td || fxl) {
      st = td ? vjp_td_sweep(c, B, nslot, s) : vjp_fxl_sweep(c, B, s);
      if (st) return st;
      tscale = 1.0 / ((double)L.cfg.num_checkpoints * (double)L.cfg.ministeps);
    } else {
      // regeneration plan (reverse order of use)
      std::vector<long> items;
      std::vector<long> item_of;
      if (!rk43) {
        for (long a = 0; a < L.nrec; ++a) {
          item_of.push_back((long)items.size());
          const long base = a * Q_NREC;
          items.push_back(base + Q_F); items.push_back(base + Q_X2); items.push_back(base + Q_X3); items.push_back(base + Q_X4);
        }
      } else {
        items.push_back(RR_X0);
        for (long a = 0; a < L.nrec; ++a) {
          if (!L.acc[a]) { item_of.push_back(-1); continue; }
          item_of.push_back((long)items.size());
          const long base = a * RR_NREC;
          items.push_back(base + RR_Y2); items.push_back(base + RR_Y3); items.push_back(base + RR_Y4); items.push_back(base + RR_XF);
        }
      }
      st = upload_items(c, items, s);
      if (st) return st;
      const long ci = (long)chunk_items(c);
      long chunk_lo = -1;
      auto phys_of = [&](long item) -> const R* {   // chunks end at the requested item (reverse sweep)
        if (chunk_lo < 0 || item < chunk_lo || item >= chunk_lo + ci) {
          chunk_lo = std::max<long>(0, item - ci + 1);
          const long cnt = std::min<long>(ci, (long)items.size() - chunk_lo);
          launch_regen<R, N>(c, (const cplx<R>*)L.rec, c->items + chunk_lo, (int)cnt, s);
        }
        return (const R*)c->Phys + (size_t)(item - chunk_lo) * N * NPH * N;
      };
      const cplx<R>* rec = (const cplx<R>*)L.rec;
      if (!rk43) {
        tscale = 1.0 / ((double)L.cfg.num_checkpoints * (double)L.cfg.ministeps);
        const double h = L.h;
        const long kseg = L.seg ? L.seg : L.nrec;
        const long nseg = (L.nrec + kseg - 1) / kseg;
        // Checkpointed record: segment g-1 is recomputed (batch 1, on the primal
        // stream with its own scratch, into the other of two record buffers)
        // while the adjoint sweeps segment g on the caller's stream.
        const bool pipe = L.seg && nseg > 1;
        if (pipe) {
          st = ensure_pipeline(c, kseg);
          if (!st) st = grow(c, &L.rec2, &L.rec2_bytes, (size_t)kseg * Q_NREC * vb);
          if (st) return st;
          cudaError_t e = cudaEventRecord(c->pev[0], s);
          if (e == cudaSuccess) e = cudaStreamWaitEvent(c->pstream, c->pev[0], 0);
          if (e != cudaSuccess) return cuda_err(c, e, "pipeline fork");
        }
        void* bufs[2] = {L.rec, L.rec2};
        auto recompute = [&](long g) -> cudaError_t {   // on the primal stream, into bufs[g & 1]
          void* const Gs = c->G; void* const Hs = c->H;
          c->G = c->Gp; c->H = c->Hp;
          rk4_segment_record(c, g * kseg, std::min(kseg, L.nrec - g * kseg), c->pstream, bufs[g & 1]);
          c->G = Gs; c->H = Hs;
          return cudaEventRecord(c->pev[g & 1], c->pstream);
        };
        if (pipe) {
          const cudaError_t e = recompute(nseg - 1);
          if (e != cudaSuccess) return cuda_err(c, e, "segment recomputation");
        }
        for (long g = nseg - 1; g >= 0; --g) {
          const long a0 = g * kseg, cnt = std::min(kseg, L.nrec - a0);
          const cplx<R>* rseg;
          if (pipe) {
            cudaError_t e = cudaSuccess;
            if (g > 0) {   // the buffer of segment g-1 was last read by the adjoint of segment g+1
              if (g + 1 < nseg) e = cudaStreamWaitEvent(c->pstream, c->tjoin[0][(g + 1) & 1], 0);
              if (e == cudaSuccess) e = recompute(g - 1);
            }
            if (e == cudaSuccess) e = cudaStreamWaitEvent(s, c->pev[g & 1], 0);
            if (e != cudaSuccess) return cuda_err(c, e, "segment recomputation");
            rseg = (const cplx<R>*)bufs[g & 1];
          } else {
            rseg = rk4_segment_record(c, a0, cnt, s);
          }
          std::vector<long> sitems;
          for (long it = 0; it < cnt; ++it) {
            const long base = it * Q_NREC;
            sitems.push_back(base + Q_F); sitems.push_back(base + Q_X2); sitems.push_back(base + Q_X3); sitems.push_back(base + Q_X4);
          }
          st = upload_items(c, sitems, s);
          if (st) return st;
          long slo = -1;
          auto sphys = [&](long item) -> const R* {   // chunks end at the requested item (reverse sweep)
            if (slo < 0 || item < slo || item >= slo + ci) {
              slo = std::max<long>(0, item - ci + 1);
              launch_regen<R, N>(c, rseg, c->items + slo, (int)std::min<long>(ci, (long)sitems.size() - slo), s);
            }
            return (const R*)c->Phys + (size_t)(item - slo) * N * NPH * N;
          };
          // seed the segment's last step from obar (J_OB)
          launch_col_adj<R, N>(c, B, AJ_PRE, rseg + (size_t)(cnt - 1) * Q_NREC * VEC, nullptr, 0.0, h, nslot, s);
          for (long it = cnt - 1; it >= 0; --it) {
            const cplx<R>* ra = rseg + (size_t)it * Q_NREC * VEC;
            const cplx<R>* rp = it > 0 ? rseg + (size_t)(it - 1) * Q_NREC * VEC : nullptr;
            for (int k = 4; k >= 1; --k) {
              launch_row_adj<R, N>(c, B, sphys(4 * it + (k - 1)), s);
              launch_col_adj<R, N>(c, B, k, ra, rp, 0.0, h, nslot, s);
            }
          }
          if (pipe) {   // the adjoint of segment g is done with bufs[g & 1]
            const cudaError_t e = cudaEventRecord(c->tjoin[0][g & 1], s);
            if (e != cudaSuccess) return cuda_err(c, e, "segment recomputation");
          }
        }
      } else {
        tscale = 1.0;
        const double t = L.T;
        for (long a = L.nrec - 1; a >= 0; --a) {
          const cplx<R>* ra = rec + (size_t)a * RR_NREC * VEC;
          const double h = L.hs[a];
          if (!L.acc[a]) {
            const int cols = B * K;
            ++c->launches; k_adj_reject<R><<<(cols + 3) / 4, 128, 0, s>>>((cplx<R>*)c->D, nslot, ra, c->hacc, N, B);
            continue;
          }
          launch_col_adj<R, N>(c, B, AJ43_PRE, ra, nullptr, t, h, nslot, s);
          for (int k = 3; k >= 0; --k) {
            launch_row_adj<R, N>(c, B, phys_of(item_of[a] + k), s);
            launch_col_adj<R, N>(c, B, AJ43_S2 + k, ra, nullptr, t, h, nslot, s);
          }
        }
        launch_col_adj<R, N>(c, B, AJ43_IPRE, rec, nullptr, t, 0.0, nslot, s);
        launch_row_adj<R, N>(c, B, phys_of(0), s);
        launch_col_adj<R, N>(c, B, AJ43_INIT, rec, nullptr, t, 0.0, nslot, s);
      }
    }
    // tail: gfields = c_fields + to_box^T(fbar0) [- (I - proj) P_sym c_fields] + phase terms
    ++c->launches; k_box_to_fields_adj<R><<<grid1d((long)B * VEC), 256, 0, s>>>(
        (const cplx<R>*)c->D + (size_t)fslot * VEC, (long)nslot * VEC, (cplx<R>*)c->V, N, B);
    launch_col_from_box<R, N>(c, (const cplx<R>*)c->V, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, gfields, cfields, nullptr, B, 2, s);
    if (carry_mode(L.mode)) {
      // tmp = P_sym c  (k_sub_sym_phys computes out -= P_sym(rest); start from zero)
      cudaMemsetAsync(c->fields_tmp, 0, (size_t)B * 2 * N * N * sizeof(R), s);
      ++c->launches; k_sub_sym_phys<R><<<grid1d((long)B * 2 * N * N), 256, 0, s>>>((R*)c->fields_tmp, cfields, odd, L.cfg.rot, N, B);
      // fields_tmp = -P c ; (I - proj)(-P c) = fields_tmp - from_box(to_box(fields_tmp)); g += that
      launch_row_to_box<R, N>(c, (const R*)c->fields_tmp, (cplx<R>*)c->H, B, s);
      launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->OUT, B, 2, s);
      launch_col_from_box<R, N>(c, (const cplx<R>*)c->OUT, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
      launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, (R*)c->fields_tmp2, (const R*)c->fields_tmp, nullptr, B, 1, s);
      ++c->launches; k_axpy<R><<<grid1d((long)B * 2 * N * N), 256, 0, s>>>(gfields, (const R*)c->fields_tmp2, R(1), (long)B * 2 * N * N);
    }
    ++c->launches; k_adj_phase<R><<<grid1d((long)B * 2 * N * N), 256, 0, s>>>(gfields, (const R*)L.vt, (const R*)L.vx, cT, csx, N, B);
    ++c->launches; k_reduce_hacc<<<(B + 127) / 128, 128, 0, s>>>(c->hacc, K, tscale, gT, B);
    return cuda_err(c, cudaGetLastError(), "vjp");
  }


  // ---------------------------------------------------------------------
  // Slot pool: continuous batching of fixed-step forward shootings.  Every
  // slot has its own step size and step budget; finished or empty slots are
  // skipped; requests are admitted between advance calls (step boundaries).
  // ---------------------------------------------------------------------
  static int pool_reset(ecs_ctx* c, cudaStream_t s) {
    ++c->launches; k_pool_init<<<(c->max_batch + 127) / 128, 128, 0, s>>>(c->ctl, 0, c->max_batch, 0);
    c->pool.assign(c->max_batch, ecs_ctx::PoolSlot());
    return cuda_err(c, cudaGetLastError(), "pool_reset");
  }

  static int pool_admit(ecs_ctx* c, int slot, const ecs_shoot_cfg* cfg, const R* fields, double T, double sx,
                        cudaStream_t s) {
    if ((int)c->pool.size() != c->max_batch) { int st = pool_reset(c, s); if (st) return st; }
    if (cfg->mode != ECS_MODE_LAWSON_RK4) return set_err(c, ECS_ERR_BAD_MODE, "the slot pool runs Lawson_RK4");
    const long steps = (long)cfg->num_checkpoints * cfg->ministeps;
    if (steps <= 0) return set_err(c, ECS_ERR_INVALID, "steps must be > 0");
    const size_t VEC = 2UL * K * M, fe = 2UL * N * N;
    R* pf = (R*)c->pool_fields + (size_t)slot * fe;
    cudaError_t e = cudaMemcpyAsync(pf, fields, fe * sizeof(R), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_err(c, e, "pool admit copy");
    launch_row_to_box<R, N>(c, pf, (cplx<R>*)c->H, 1, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->F + (size_t)slot * VEC, 1, 2, s);
    ++c->launches; k_fill<<<1, 32, 0, s>>>(c->Tbuf + slot, T, 1);
    ++c->launches; k_fill<<<1, 32, 0, s>>>(c->pool_sx + slot, sx, 1);
    ++c->launches;
    k_rk4_setup<R><<<grid1d((long)VEC), 256, 0, s>>>(c->Tbuf + slot, cfg->num_checkpoints, cfg->ministeps,
                                                     c->ctl + slot, (R*)c->Etab + (size_t)slot * VEC, N, c->nu,
                                                     c->eta, 1);
    ++c->launches; k_pool_init<<<1, 32, 0, s>>>(c->ctl, slot, 1, (int)steps);
    auto& ps = c->pool[slot];
    ps.active = 1; ps.ny = cfg->shift_reflect_ny; ps.rot = cfg->rot; ps.steps = steps;
    return cuda_err(c, cudaGetLastError(), "pool_admit");
  }

  static int pool_advance(ecs_ctx* c, int nsteps, cudaStream_t s) {
    const int B = c->max_batch;
    auto one_step = [&](cudaStream_t st_) {
      for (int st = 1; st <= 4; ++st) {
        launch_row_rhs<R, N>(c, B, st_, c->ctl);
        launch_col_rk4<R, N>(c, B, st, 1, 0, st_, nullptr, 0, 1);
      }
      ++c->launches; k_pool_count<<<(B + 127) / 128, 128, 0, st_>>>(c->ctl, B);
    };
    constexpr int GS = 8;
    auto& gk = c->gpool;
    if (!gk.exec) {
      const long long l0 = c->launches;
      cudaGraph_t graph = nullptr;
      std::lock_guard<std::mutex> capture_guard(capture_mutex());   // no set-up of another context meanwhile
      cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int a = 0; a < GS; ++a) one_step(c->cap_stream);
        e = cudaStreamEndCapture(c->cap_stream, &graph);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&gk.exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) { gk.exec = nullptr; return cuda_err(c, e, "pool graph capture"); }
      gk.nodes = c->launches - l0;
      c->launches = l0;
    }
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s, nullptr, 0, 1);
    int it = 0;
    for (; it + GS <= nsteps; it += GS) {
      cudaError_t e = cudaGraphLaunch(gk.exec, s);
      if (e != cudaSuccess) return cuda_err(c, e, "pool graph launch");
      c->launches += gk.nodes;
    }
    for (; it < nsteps; ++it) one_step(s);
    return cuda_err(c, cudaGetLastError(), "pool_advance");
  }

  static int pool_retire(ecs_ctx* c, int slot, R* out_fields, double* loss, cudaStream_t s) {
    const size_t VEC = 2UL * K * M, fe = 2UL * N * N;
    auto& ps = c->pool[slot];
    const R* pf = (const R*)c->pool_fields + (size_t)slot * fe;
    launch_col_from_box<R, N>(c, (const cplx<R>*)c->F + (size_t)slot * VEC, (cplx<R>*)c->G, 1, c->pool_sx + slot,
                              ps.ny, ps.rot, 1, 0, s, 1);
    R* out = out_fields ? out_fields : (R*)c->fields_tmp;
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, out, pf, nullptr, 1, 1, s);
    if (loss) {
      ++c->launches; k_rowsq<R><<<N, 32, 0, s>>>(out, c->rowsq, N);
      ++c->launches; k_reduce_rows<<<1, 128, 0, s>>>(c->rowsq, loss, N, 1, 1.0 / (2.0 * N * N));
    }
    ps.active = 0;
    ++c->launches; k_pool_init<<<1, 32, 0, s>>>(c->ctl, slot, 1, 0);
    return cuda_err(c, cudaGetLastError(), "pool_retire");
  }

  // ---------------------------------------------------------------------
  // Several candidates' Lawson-RK4 objectives and one JVP each, in one
  // forward-mode sweep (ecs_jvp_multi): B independent jax.jvp calls of
  // objective_RPO (jax_scripts/lib/utils.py:108) batched across candidates.
  // The B primal solves step together as the slot pool's do (own T, h,
  // symmetry, step budget per candidate: control block b), and each stage's
  // tangent pass follows that stage's primal pass: the primal row pass writes
  // the stage's physical fields u, v, B_x, B_y per candidate, the primal
  // column pass the step's record vectors (one step, overwritten each step),
  // and the tangent row and column passes read them.  Nothing else is kept,
  // so device memory does not grow with the horizon.  A candidate whose budget
  // is spent is skipped by every later launch.  Steps run as 8-step CUDA
  // graphs (per-candidate data is read from the control blocks).
  // ---------------------------------------------------------------------
  static int ensure_multi(ecs_ctx* c) {
    auto& m = c->mj;
    if (m.G) return ECS_OK;
    const size_t B = (size_t)c->max_batch, VEC = 2UL * K * M, cb = sizeof(cplx<R>), rb = sizeof(R);
    int st = ECS_OK;
    m.G = dev_alloc(c, B * NG * K * N * cb, &st);
    m.H = dev_alloc(c, B * NH * K * N * cb, &st);
    m.phys = dev_alloc(c, B * N * NPH * N * rb, &st);
    m.rec = dev_alloc(c, B * Q_NREC * VEC * cb, &st);
    m.vt = dev_alloc(c, B * 2 * N * N * rb, &st);
    m.vx = dev_alloc(c, B * 2 * N * N * rb, &st);
    m.dscale = (double*)dev_alloc(c, B * sizeof(double), &st);
    m.dT = (double*)dev_alloc(c, B * sizeof(double), &st);
    return st;
  }

  static int jvp_multi(ecs_ctx* c, const ecs_shoot_cfg* cfgs, const R* fields, const double* T, const double* sx,
                       R* out_fields, const R* dfields, const double* dT, const double* dsx, R* out, double* odT,
                       double* odsx, int B, cudaStream_t s) {
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>), fe = 2UL * N * N;
    const long pstride = (long)N * NPH * N, rstride = (long)Q_NREC * VEC;
    const int nslot = (int)D_NS4;
    std::vector<double> dscale(B);
    long smax = 0;
    for (int b = 0; b < B; ++b) {
      if (cfgs[b].mode != ECS_MODE_LAWSON_RK4) return set_err(c, ECS_ERR_BAD_MODE, "ecs_jvp_multi runs Lawson_RK4");
      const long steps = (long)cfgs[b].num_checkpoints * cfgs[b].ministeps;
      if (cfgs[b].num_checkpoints <= 0 || cfgs[b].ministeps <= 0 || steps > (1L << 30))
        return set_err(c, ECS_ERR_INVALID, "num_checkpoints and ministeps must be > 0");
      smax = std::max(smax, steps);
      dscale[b] = 1.0 / ((double)cfgs[b].num_checkpoints * (double)cfgs[b].ministeps);
    }
    int st = ensure_multi(c);
    if (!st) st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (st) return st;
    auto& m = c->mj;
    c->pool.clear();   // the control blocks are reused: a slot pool on this context starts over
    cudaError_t e = cudaMemcpyAsync(m.dscale, dscale.data(), B * sizeof(double), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(m.dT, dT, B * sizeof(double), cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return cuda_err(c, e, "jvp_multi scales");
    dT = m.dT;   // the captured steps read the context's copy
    // primal and tangent start states (boxes of rfft2(fields), rfft2(dfields))
    st = to_box(c, fields, (cplx<R>*)c->F, B, s);
    if (st) return st;
    launch_row_to_box<R, N>(c, dfields, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->D + (size_t)D_F * VEC, B, 2, s, (long)nslot * VEC);
    // per candidate: h = (T/nc)/ms, e = exp(h/2 L) mask, step budget
    for (int b = 0; b < B; ++b) {
      ++c->launches;
      k_rk4_setup<R><<<grid1d((long)VEC), 256, 0, s>>>(T + b, cfgs[b].num_checkpoints, cfgs[b].ministeps, c->ctl + b,
                                                       (R*)c->Etab + (size_t)b * VEC, N, c->nu, c->eta, 1);
      ++c->launches;
      k_pool_init<<<1, 32, 0, s>>>(c->ctl, b, 1, (int)((long)cfgs[b].num_checkpoints * cfgs[b].ministeps));
    }
    // phase fields (stop-gradient, loss_functions.py:113-130): vt = irfft2(state_vel(f0)), vx = irfft2(i kx f0)
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s);
    launch_row_rhs<R, N>(c, B, s);
    launch_col_rk4<R, N>(c, B, COL_PLAIN, 0, 1, s);
    st = from_box(c, (const cplx<R>*)c->OUT, (R*)m.vt, B, s);
    if (st) return st;
    launch_col_from_box<R, N>(c, (const cplx<R>*)c->F, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 1, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, (R*)m.vx, nullptr, nullptr, B, 0, s);
    // the sweep: per stage, the primal pass on (G, H), then the tangent pass on the tangents' (G, H)
    void* const G0 = c->G; void* const H0 = c->H;
    auto tangent_bufs = [&](bool on) { c->G = on ? m.G : G0; c->H = on ? m.H : H0; };
    auto start = [&](cudaStream_t st_) {
      launch_col_rk4<R, N>(c, B, COL_START, 1, 0, st_, nullptr, 0, 1);
      tangent_bufs(true);
      launch_col_tan<R, N>(c, B, TS_START, 1, (const cplx<R>*)m.rec, dT, 0.0, 0.0, 0.0, nslot, st_, c->ctl, rstride,
                           m.dscale, (const R*)c->Etab);
      tangent_bufs(false);
    };
    auto one_step = [&](cudaStream_t st_) {
      for (int q = 1; q <= 4; ++q) {
        launch_row_rhs<R, N>(c, B, st_, c->ctl, (R*)m.phys, pstride);
        launch_col_rk4<R, N>(c, B, q, 1, 0, st_, (cplx<R>*)m.rec, rstride, 1);
        tangent_bufs(true);
        launch_row_tan<R, N>(c, B, (const R*)m.phys, st_, pstride, c->ctl);
        launch_col_tan<R, N>(c, B, q, 1, (const cplx<R>*)m.rec, dT, 0.0, 0.0, 0.0, nslot, st_, c->ctl, rstride,
                             m.dscale, (const R*)c->Etab);
        tangent_bufs(false);
      }
      ++c->launches; k_pool_count<<<(B + 127) / 128, 128, 0, st_>>>(c->ctl, B);
    };
    constexpr int GS = 8;
    auto& gk = m.g;
    if (gk.exec && (gk.B != B || gk.D != c->D)) { cudaGraphExecDestroy(gk.exec); gk.exec = nullptr; }
    if (!gk.exec && smax >= GS) {
      const long long l0 = c->launches;
      cudaGraph_t graph = nullptr;
      std::lock_guard<std::mutex> capture_guard(capture_mutex());   // no set-up of another context meanwhile
      e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        for (int a = 0; a < GS; ++a) one_step(c->cap_stream);
        e = cudaStreamEndCapture(c->cap_stream, &graph);
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&gk.exec, graph, 0);
      if (graph) cudaGraphDestroy(graph);
      if (e != cudaSuccess) { gk.exec = nullptr; return cuda_err(c, e, "jvp_multi graph capture"); }
      gk.B = B; gk.D = c->D;
      gk.nodes = c->launches - l0;
      c->launches = l0;
    }
    start(s);
    long it = 0;
    for (; gk.exec && it + GS <= smax; it += GS) {
      e = cudaGraphLaunch(gk.exec, s);
      if (e != cudaSuccess) return cuda_err(c, e, "jvp_multi graph launch");
      c->launches += gk.nodes;
    }
    for (; it < smax; ++it) one_step(s);
    // per candidate: objective residual, tangent residual, phase-condition tangents
    for (int b = 0; b < B; ++b) {
      const cplx<R>* phi = (const cplx<R>*)c->F + (size_t)b * VEC;
      if (out_fields) {
        st = residual(c, &cfgs[b], fields + (size_t)b * fe, phi, nullptr, sx + b, 1, out_fields + (size_t)b * fe, s, 1);
        if (st) return st;
      }
      ++c->launches;
      k_tan_shift<R><<<grid1d((long)VEC), 256, 0, s>>>((const cplx<R>*)c->D + ((size_t)b * nslot + D_F) * VEC,
                                                       (long)nslot * VEC, phi, dsx + b, (cplx<R>*)c->V, N, 1);
      st = residual(c, &cfgs[b], dfields + (size_t)b * fe, (const cplx<R>*)c->V, nullptr, sx + b, 1,
                    out + (size_t)b * fe, s, 1);
      if (st) return st;
      ++c->launches;
      k_phase_dot<R><<<1, 256, 0, s>>>((const R*)m.vt + (size_t)b * fe, (const R*)m.vx + (size_t)b * fe,
                                       dfields + (size_t)b * fe, odT + b, odsx + b, N);
    }
    return cuda_err(c, cudaGetLastError(), "jvp_multi");
  }

  // ---------------------------------------------------------------------
  // Several candidates' loss_RPO and its gradient in one adjoint sweep
  // (ecs_loss_grad_multi): B independent jax.value_and_grad(loss_RPO) calls
  // (jax_scripts/adjoint_descent.py:91), Lawson_RK4.  The B forward solves step
  // together (per-candidate h, symmetry and step budget in the control
  // blocks), keeping each candidate's state every SEG steps (SEG divides every
  // candidate's step count).  The reverse sweep is aligned at each candidate's
  // end: in reverse segment r candidate b recomputes its segment
  // nseg_b - 1 - r from its checkpoint (with the record and the stage fields
  // of all SEG steps kept), then the adjoint passes sweep it backwards;
  // candidates without such a segment are skipped.  Loss mean(out^2) over
  // 2 n^2 entries, cotangent out / n^2 (loss_functions.py:99-111).
  // ---------------------------------------------------------------------
  static int loss_grad_multi(ecs_ctx* c, const ecs_shoot_cfg* cfgs, const R* fields, const double* T,
                             const double* sx, double* loss, R* gfields, double* gT, double* gsx, int B,
                             cudaStream_t s) {
    const size_t VEC = 2UL * K * M, vb = VEC * sizeof(cplx<R>), fe = 2UL * N * N;
    const long pstride = (long)N * NPH * N;
    const int nslot = (int)J_NS4;
    std::vector<long> steps(B);
    std::vector<int> nseg(B);
    long smax = 0, seg = 0;
    for (int b = 0; b < B; ++b) {
      if (cfgs[b].mode != ECS_MODE_LAWSON_RK4) return set_err(c, ECS_ERR_BAD_MODE, "ecs_loss_grad_multi runs Lawson_RK4");
      steps[b] = (long)cfgs[b].num_checkpoints * cfgs[b].ministeps;
      if (cfgs[b].num_checkpoints <= 0 || cfgs[b].ministeps <= 0 || steps[b] > (1L << 30))
        return set_err(c, ECS_ERR_INVALID, "num_checkpoints and ministeps must be > 0");
      smax = std::max(smax, steps[b]);
      seg = std::gcd(seg, steps[b]);
    }
    seg = std::min(seg, 32L);
    while (seg > 1) {   // SEG must divide every step count
      bool ok = true;
      for (int b = 0; b < B; ++b) ok = ok && steps[b] % seg == 0;
      if (ok) break;
      --seg;
    }
    for (int b = 0; b < B; ++b) nseg[b] = (int)(steps[b] / seg);
    const long nsegmax = smax / seg;
    int st = ensure_multi(c);
    auto& m = c->mj;
    if (!st) st = grow(c, &c->D, &c->D_bytes, (size_t)B * nslot * vb);
    if (!st) st = grow(c, (void**)&c->hacc, &c->hacc_bytes, (size_t)B * K * 2 * sizeof(double));
    if (!st) st = grow(c, &m.ckpt, &m.ckpt_bytes, (size_t)nsegmax * B * vb);
    if (!st) st = grow(c, &m.grec, &m.grec_bytes, (size_t)B * seg * Q_NREC * vb);
    if (!st) st = grow(c, &m.gphys, &m.gphys_bytes, (size_t)seg * 4 * B * pstride * sizeof(R));
    if (!st) st = grow(c, &m.res, &m.res_bytes, (size_t)2 * B * fe * sizeof(R));
    if (!st && !m.nseg) m.nseg = (int*)dev_alloc(c, (size_t)c->max_batch * sizeof(int), &st);
    if (st) return st;
    c->pool.clear();   // the control blocks are reused: a slot pool on this context starts over
    cudaError_t e = cudaMemcpyAsync(m.nseg, nseg.data(), B * sizeof(int), cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return cuda_err(c, e, "loss_grad_multi segments");
    cplx<R>* F = (cplx<R>*)c->F;
    st = to_box(c, fields, F, B, s);
    if (st) return st;
    for (int b = 0; b < B; ++b) {
      ++c->launches;
      k_rk4_setup<R><<<grid1d((long)VEC), 256, 0, s>>>(T + b, cfgs[b].num_checkpoints, cfgs[b].ministeps, c->ctl + b,
                                                       (R*)c->Etab + (size_t)b * VEC, N, c->nu, c->eta, 1);
      ++c->launches; k_pool_init<<<1, 32, 0, s>>>(c->ctl, b, 1, (int)steps[b]);
    }
    // forward solves with a checkpoint every SEG steps (the loss has no phase-condition part)
    cplx<R>* ckpt = (cplx<R>*)m.ckpt;
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s, nullptr, 0, 1);
    for (long it = 0; it < smax; ++it) {
      if (it % seg == 0) {
        e = cudaMemcpyAsync(ckpt + (size_t)(it / seg) * B * VEC, F, B * vb, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_err(c, e, "loss_grad_multi checkpoint");
      }
      for (int q = 1; q <= 4; ++q) {
        launch_row_rhs<R, N>(c, B, s, c->ctl);
        launch_col_rk4<R, N>(c, B, q, 1, 0, s, nullptr, 0, 1);
      }
      ++c->launches; k_pool_count<<<(B + 127) / 128, 128, 0, s>>>(c->ctl, B);
    }
    // residuals out_b = fields_b - irfft2(sym(shift(phi_b))), losses, cotangents out_b / n^2
    R* res = (R*)m.res;
    R* cot = res + (size_t)B * fe;
    for (int b = 0; b < B; ++b) {
      st = residual(c, &cfgs[b], fields + (size_t)b * fe, F + (size_t)b * VEC, nullptr, sx + b, 1, res + (size_t)b * fe,
                    s, 1);
      if (st) return st;
      ++c->launches; k_rowsq<R><<<N, 32, 0, s>>>(res + (size_t)b * fe, c->rowsq, N);
      ++c->launches; k_reduce_rows<<<1, 128, 0, s>>>(c->rowsq, loss + b, N, 1, 1.0 / (2.0 * N * N));
    }
    e = cudaMemsetAsync(cot, 0, B * fe * sizeof(R), s);   // cot = res / n^2 (exact: n^2 is a power of two)
    if (e != cudaSuccess) return cuda_err(c, e, "loss_grad_multi cotangent");
    ++c->launches; k_axpy<R><<<grid1d((long)B * fe), 256, 0, s>>>(cot, res, R(1) / (R(N) * R(N)), (long)B * fe);
    // head: Ybar = -(c/n^2) rfft2(cot) on the box; Phibar = sym^T(Ybar) and sxbar per candidate
    cudaMemsetAsync(c->D, 0, (size_t)B * nslot * vb, s);
    cudaMemsetAsync(c->hacc, 0, (size_t)B * K * 2 * sizeof(double), s);
    launch_row_to_box<R, N>(c, cot, (cplx<R>*)c->H, B, s);
    launch_col_to_box<R, N>(c, (const cplx<R>*)c->H, (cplx<R>*)c->V, B, 2, s);
    ++c->launches; k_box_scale_c<R><<<grid1d((long)B * VEC), 256, 0, s>>>((cplx<R>*)c->V, (long)VEC, N, B, R(-1) / (R(N) * R(N)));
    for (int b = 0; b < B; ++b) {
      const int odd = (cfgs[b].shift_reflect_ny % 2 + 2) % 2 == 1;
      const double sy = (cfgs[b].shift_reflect_ny * 2 * M_PI) / 8;
      ++c->launches;
      k_adj_head<R><<<1, 256, 0, s>>>((const cplx<R>*)c->V + (size_t)b * VEC, (const cplx<R>*)F + (size_t)b * VEC,
                                      sx + b, 1, sy, odd, cfgs[b].rot, (cplx<R>*)c->D + ((size_t)b * nslot + J_OB) * VEC,
                                      (long)nslot * VEC, gsx + b, N);
    }
    // reverse segments
    cplx<R>* grec = (cplx<R>*)m.grec;
    R* gphys = (R*)m.gphys;
    const long rstride = (long)seg * Q_NREC * VEC;
    for (long r = 0; r < nsegmax; ++r) {
      ++c->launches;
      k_grad_segment<R><<<grid1d((long)B * VEC), 256, 0, s>>>(F, ckpt, m.nseg, (int)r, c->ctl, (long)VEC, B);
      launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s, nullptr, 0, 1);
      for (long it = 0; it < seg; ++it) {
        for (int q = 1; q <= 4; ++q) {
          launch_row_rhs<R, N>(c, B, s, c->ctl, gphys + (size_t)(it * 4 + q - 1) * B * pstride, pstride);
          launch_col_rk4<R, N>(c, B, q, (q == 4 && it == seg - 1) ? 0 : 1, 0, s, grec + (size_t)it * Q_NREC * VEC,
                               rstride, 1);
        }
      }
      launch_col_adj<R, N>(c, B, AJ_PRE, grec + (size_t)(seg - 1) * Q_NREC * VEC, nullptr, 0.0, 0.0, nslot, s,
                           c->ctl, rstride);
      for (long it = seg - 1; it >= 0; --it) {
        const cplx<R>* ra = grec + (size_t)it * Q_NREC * VEC;
        const cplx<R>* rp = it > 0 ? grec + (size_t)(it - 1) * Q_NREC * VEC : nullptr;
        for (int k = 4; k >= 1; --k) {
          launch_row_adj<R, N>(c, B, gphys + (size_t)(it * 4 + k - 1) * B * pstride, s, pstride, c->ctl);
          launch_col_adj<R, N>(c, B, k, ra, rp, 0.0, 0.0, nslot, s, c->ctl, rstride);
        }
      }
    }
    // tail per candidate: gfields = cot + to_box^T(fbar0) + phase terms; gT from the h accumulators
    ++c->launches; k_box_to_fields_adj<R><<<grid1d((long)B * VEC), 256, 0, s>>>(
        (const cplx<R>*)c->D + (size_t)J_OB * VEC, (long)nslot * VEC, (cplx<R>*)c->V, N, B);
    launch_col_from_box<R, N>(c, (const cplx<R>*)c->V, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, gfields, cot, nullptr, B, 2, s);
    for (int b = 0; b < B; ++b) {
      const double tscale = 1.0 / ((double)cfgs[b].num_checkpoints * (double)cfgs[b].ministeps);
      ++c->launches; k_reduce_hacc<<<1, 128, 0, s>>>(c->hacc + (size_t)b * K * 2, K, tscale, gT + b, 1);
    }
    return cuda_err(c, cudaGetLastError(), "loss_grad_multi");
  }

  // Time `iters` launches of one hot kernel on the current workspace (after a
  // jvp call) with CUDA events on stream s; returns ms per launch and the
  // kernel's algorithmic bytes per launch.
  static int bench_kernel(ecs_ctx* c, int which, int B, int iters, float* ms, double* bytes, cudaStream_t s) {
    auto& L = c->lin;
    if (!L.valid || !c->Phys || !c->D) return set_err(c, ECS_ERR_INVALID, "bench_kernel needs a prior ecs_jvp call");
    const size_t VEC = 2UL * K * M, cb = sizeof(cplx<R>), rb = sizeof(R);
    const bool rk43 = L.mode == ECS_MODE_LAWSON_RK43;
    const int nslot = rk43 ? (int)S_NSLOT : (int)D_NS4;
    cudaMemsetAsync(c->Tbuf, 0, sizeof(double) * B, s);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0); cudaEventCreate(&e1);
    auto launch = [&]() {
      if (which == 0) launch_row_tan<R, N>(c, B, (const R*)c->Phys, s);
      else if (rk43) launch_col_tan<R, N>(c, B, T43_B, 1, (const cplx<R>*)L.rec, c->Tbuf, L.T, L.h, 1.0, nslot, s);
      else launch_col_tan<R, N>(c, B, T4_S2, 1, (const cplx<R>*)L.rec, c->Tbuf, 0.0, L.h, 1.0, nslot, s);
    };
    launch();
    cudaEventRecord(e0, s);
    for (int i = 0; i < iters; ++i) launch();
    cudaEventRecord(e1, s);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0; cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0); cudaEventDestroy(e1);
    if (e != cudaSuccess) return cuda_err(c, e, "bench_kernel");
    *ms = t / iters;
    if (which == 0) *bytes = (double)B * (NG + NH) * K * N * cb + (double)N * NPH * N * rb;
    else *bytes = (double)B * (NH * K * N * cb + NG * K * N * cb + 2 * VEC * cb) + (double)VEC * cb;
    return ECS_OK;
  }
};

}  // namespace ecs

namespace ecs {
template <typename R, int N>
int ctx_init(ecs_ctx* c, const ecs_params* prm) {
  int st = configure_kernels<R, N>(c);
  if (st) return st;
  const int B = c->max_batch;
  const size_t cb = sizeof(cplx<R>), rb = sizeof(R);
  const size_t nbox = (size_t)B * 2 * Geomc<N>::K * Geomc<N>::M;
  c->F = dev_alloc(c, nbox * cb, &st);
  c->A1 = dev_alloc(c, nbox * cb, &st);
  c->K2 = dev_alloc(c, nbox * cb, &st);
  c->OUT = dev_alloc(c, nbox * cb, &st);
  c->V = dev_alloc(c, nbox * cb, &st);
  c->Etab = dev_alloc(c, nbox * rb, &st);
  // G holds NG (stepping) or 2 (boundary) fields, H holds NH, NHA or 2
  c->G = dev_alloc(c, (size_t)B * NG * Geomc<N>::K * N * cb, &st);
  c->H = dev_alloc(c, (size_t)B * NHA * Geomc<N>::K * N * cb, &st);
  c->fields_tmp = dev_alloc(c, (size_t)B * 2 * N * N * rb, &st);
  c->fields_tmp2 = dev_alloc(c, (size_t)B * 2 * N * N * rb, &st);
  c->S43 = dev_alloc(c, nbox * S_NSLOT * cb, &st);
  c->dcount = (int*)dev_alloc(c, sizeof(int), &st);
  c->pool_fields = dev_alloc(c, (size_t)B * 2 * N * N * rb, &st);
  c->pool_sx = (double*)dev_alloc(c, (size_t)B * sizeof(double), &st);
  c->ctl = (StepCtl*)dev_alloc(c, (size_t)B * sizeof(StepCtl), &st);
  c->rowsq = (double*)dev_alloc(c, (size_t)B * N * sizeof(double), &st);
  c->Tbuf = (double*)dev_alloc(c, (size_t)B * sizeof(double), &st);
  c->tw = dev_alloc(c, (size_t)tw_smem(N) * cb, &st);   // the shared-memory twiddle image
  c->fhat = dev_alloc(c, (size_t)Geomc<N>::K * Geomc<N>::M * cb, &st);
  if (st) return st;
  if (cudaMallocHost((void**)&c->hcount, sizeof(int)) != cudaSuccess) return set_err(c, ECS_ERR_OOM, "pinned alloc");
  if (cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking) != cudaSuccess)
    return set_err(c, ECS_ERR_CUDA, "capture stream");
  // twiddles exp(-2 pi i k/N), k < N/2, from long double
  std::vector<cplx<R>> tw(N / 2);
  const long double twopi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < N / 2; ++k) {
    long double a = twopi * (long double)k / (long double)N;
    tw[k] = mk<R>((R)cosl(a), (R)(-sinl(a)));
  }
  std::vector<cplx<R>> img(tw_smem(N));
  twiddle_image<cplx<R>, N>(tw.data(), img.data());
  cudaError_t e = cudaMemcpy(c->tw, img.data(), img.size() * cb, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_err(c, e, "twiddle upload");
  // forcing on the grid x_i = i/n * 2 * pi (mhd_jax.py:47), channel omega only
  std::vector<R> fr((size_t)2 * N * N, R(0));
  const double pi_lit = 3.14159265358979323846;
  for (int i = 0; i < N; ++i)
    for (int jy = 0; jy < N; ++jy) {
      double v;
      if (prm->forcing) v = prm->forcing[(size_t)i * N + jy];
      else {
        const double y = (double)jy / N * 2 * pi_lit;
        v = prm->kolmogorov_amp * cos(prm->kolmogorov_k * y);
      }
      fr[(size_t)i * N + jy] = (R)v;
    }
  e = cudaMemcpy(c->fields_tmp, fr.data(), fr.size() * rb, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_err(c, e, "forcing upload");
  st = Impl<R, N>::to_box(c, (const R*)c->fields_tmp, (cplx<R>*)c->V, 1, 0);
  if (st) return st;
  // channel-omega box with mask[0,0] = False
  e = cudaMemcpy(c->fhat, c->V, (size_t)Geomc<N>::K * Geomc<N>::M * cb, cudaMemcpyDeviceToDevice);
  if (e == cudaSuccess) e = cudaMemset(c->fhat, 0, cb);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return cuda_err(c, e, "forcing spectrum");
}
}  // namespace ecs

namespace ecs {

// Function table of one (dtype, n): the C entry points dispatch through it.
template <typename R, int N>
ImplTable make_table() {
  using I = Impl<R, N>;
  ImplTable t;
  t.init = [](ecs_ctx* c, const ecs_params* p) { return ctx_init<R, N>(c, p); };
  t.to_box = [](ecs_ctx* c, const void* f, void* b, int B, cudaStream_t s) {
    return I::to_box(c, (const R*)f, (cplx<R>*)b, B, s); };
  t.from_box = [](ecs_ctx* c, const void* b, void* f, int B, cudaStream_t s) {
    return I::from_box(c, (const cplx<R>*)b, (R*)f, B, s); };
  t.dealias = [](ecs_ctx* c, const void* f, void* o, int B, cudaStream_t s) {
    return I::dealias(c, (const R*)f, (R*)o, B, s); };
  t.state_vel = [](ecs_ctx* c, const void* f, void* o, int B, int d, cudaStream_t s) {
    return I::state_vel(c, (const cplx<R>*)f, (cplx<R>*)o, B, d, s); };
  t.lawson_rk4 = [](ecs_ctx* c, void* f, double t_, int st, int B, cudaStream_t s) {
    return I::lawson_rk4(c, (cplx<R>*)f, t_, st, B, s); };
  t.shoot = [](ecs_ctx* c, const ecs_shoot_cfg* cfg, const void* f, const double* T, const double* sx, void* o,
               double* loss, ecs_info* info, int B, cudaStream_t s) {
    return I::shoot(c, cfg, (const R*)f, T, sx, (R*)o, loss, info, B, s); };
  t.linearize = [](ecs_ctx* c, const ecs_shoot_cfg* cfg, const void* f, const double* T, const double* sx, void* o,
                   ecs_info* info, cudaStream_t s) {
    return I::linearize(c, cfg, (const R*)f, T, sx, (R*)o, info, s); };
  t.jvp = [](ecs_ctx* c, const void* df, const double* dT, const double* dsx, void* o, double* oT, double* osx, int B,
             cudaStream_t s) { return I::jvp(c, (const R*)df, dT, dsx, (R*)o, oT, osx, B, s); };
  t.integrate = [](ecs_ctx* c, int mode, void* f, double t_, int steps, int B, cudaStream_t s) {
    return I::integrate_mode(c, mode, (cplx<R>*)f, t_, steps, B, s); };
  t.recurrence = [](ecs_ctx* c, const void* fs, int S, double* dist, cudaStream_t s) {
    return I::recurrence(c, (const cplx<R>*)fs, S, dist, s); };
  t.linearize_jvp = [](ecs_ctx* c, const ecs_shoot_cfg* cfg, const void* f, const double* T, const double* sx, void* o,
                       ecs_info* info, const void* df, const double* dT, const double* dsx, void* od, double* oT,
                       double* osx, int B, cudaStream_t s) {
    return I::linearize_jvp(c, cfg, (const R*)f, T, sx, (R*)o, info, (const R*)df, dT, dsx, (R*)od, oT, osx, B, s); };
  t.vjp = [](ecs_ctx* c, const void* cf, const double* cT, const double* csx, void* g, double* gT, double* gsx, int B,
             cudaStream_t s) { return I::vjp(c, (const R*)cf, cT, csx, (R*)g, gT, gsx, B, s); };
  t.bench_kernel = [](ecs_ctx* c, int which, int B, int iters, float* ms, double* bytes, cudaStream_t s) {
    return I::bench_kernel(c, which, B, iters, ms, bytes, s); };
  t.jvp_multi = [](ecs_ctx* c, const ecs_shoot_cfg* cfgs, const void* f, const double* T, const double* sx, void* o,
                   const void* df, const double* dT, const double* dsx, void* od, double* oT, double* osx, int B,
                   cudaStream_t s) {
    return I::jvp_multi(c, cfgs, (const R*)f, T, sx, (R*)o, (const R*)df, dT, dsx, (R*)od, oT, osx, B, s); };
  t.loss_grad_multi = [](ecs_ctx* c, const ecs_shoot_cfg* cfgs, const void* f, const double* T, const double* sx,
                         double* loss, void* g, double* gT, double* gsx, int B, cudaStream_t s) {
    return I::loss_grad_multi(c, cfgs, (const R*)f, T, sx, loss, (R*)g, gT, gsx, B, s); };
  t.pool_reset = [](ecs_ctx* c, cudaStream_t s) { return I::pool_reset(c, s); };
  t.pool_admit = [](ecs_ctx* c, int slot, const ecs_shoot_cfg* cfg, const void* f, double T, double sx,
                    cudaStream_t s) { return I::pool_admit(c, slot, cfg, (const R*)f, T, sx, s); };
  t.pool_advance = [](ecs_ctx* c, int nsteps, cudaStream_t s) { return I::pool_advance(c, nsteps, s); };
  t.pool_retire = [](ecs_ctx* c, int slot, void* o, double* loss, cudaStream_t s) {
    return I::pool_retire(c, slot, (R*)o, loss, s); };
  return t;
}

}  // namespace ecs
