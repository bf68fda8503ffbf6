// C ABI of the ECS-MHD-2D B200 hot path: context, workspace, dispatch and the
// host-side orchestration of the kernels in kernels.cuh.
#include "../../include/ecs_mhd.h"
#include "kernels.cuh"
#include "kernels_rk43.cuh"
#include "api_internal.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace ecs;

const char* ecs_version(void) { return "ecs_mhd_2d_b200 0.1 (sm_100a)"; }

const char* ecs_last_error(const ecs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ecs_box_dims(const ecs_ctx* ctx, int* K, int* M) {
  if (!ctx || !K || !M) return ECS_ERR_INVALID;
  *K = ctx->g.K; *M = ctx->g.M;
  return ECS_OK;
}

namespace ecs {

int set_err(ecs_ctx* c, int code, const std::string& msg) {
  if (c) c->err = msg;
  return code;
}

int cuda_err(ecs_ctx* c, cudaError_t e, const char* where) {
  if (e == cudaSuccess) return ECS_OK;
  return set_err(c, ECS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

void* dev_alloc(ecs_ctx* c, size_t bytes, int* st) {
  void* p = nullptr;
  if (*st != ECS_OK) return nullptr;
  cudaError_t e = cudaMalloc(&p, bytes < 256 ? 256 : bytes);
  if (e != cudaSuccess) {
    *st = set_err(c, ECS_ERR_OOM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    return nullptr;
  }
  c->allocs.push_back(p);
  return p;
}

}  // namespace ecs

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
namespace ecs {

constexpr int XT = 8;
constexpr int COLWARPS = 4;

template <typename R, int N> size_t smem_row_rhs() { return (N / 2 + 10 * Geomc<N>::K * (XT + 1)) * sizeof(cplx<R>); }
template <typename R, int N> size_t smem_row_2f() { return (N / 2 + 2 * Geomc<N>::K * (XT + 1)) * sizeof(cplx<R>); }

template <typename R, int N>
int configure_kernels(ecs_ctx* c) {
  int st = ECS_OK;
  st |= (int)cudaFuncSetAttribute(k_row_rhs<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_rhs<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_to_box<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_from_box<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N>());
  st |= (int)cudaFuncSetAttribute(k_row_err<R, N, XT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_row_2f<R, N>());
  if (st) return cuda_err(c, cudaGetLastError(), "cudaFuncSetAttribute");
  return ECS_OK;
}

template <typename R, int N>
void launch_row_to_box(ecs_ctx* c, const R* fields, cplx<R>* H, int B, cudaStream_t s) {
  RowFwdParams<R> p; p.fields = fields; p.H = H; p.tw = (const cplx<R>*)c->tw; p.B = B;
  k_row_to_box<R, N, XT><<<B * (N / XT), XT * 32, smem_row_2f<R, N>(), s>>>(p);
}

template <typename R, int N>
void launch_col_to_box(ecs_ctx* c, const cplx<R>* H, cplx<R>* V, int B, int nf, cudaStream_t s, long vstride = 0) {
  ColBoxParams<R> p; p.H = H; p.V = V; p.tw = (const cplx<R>*)c->tw; p.B = B; p.nf = nf;
  p.vstride = vstride > 0 ? vstride : (long)nf * Geomc<N>::K * Geomc<N>::M;
  const int cols = B * nf * Geomc<N>::K;
  k_col_to_box<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
}

template <typename R, int N>
void launch_col_from_box(ecs_ctx* c, const cplx<R>* V, cplx<R>* G2, int B, const double* sx, int ny, int rot,
                         int use_sym, int mult_ikx, cudaStream_t s) {
  ColFromBoxParams<R> p; p.V = V; p.G = G2; p.tw = (const cplx<R>*)c->tw; p.sx = sx;
  p.sy = (ny * 2 * M_PI) / 8;   // symmetry.py:11 s = (n*2*pi)/8
  p.odd = (ny % 2 + 2) % 2 == 1; p.rot = rot; p.use_sym = use_sym; p.mult_ikx = mult_ikx; p.B = B;
  const int cols = B * 2 * Geomc<N>::K;
  k_col_from_box<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
}

template <typename R, int N>
void launch_row_from_box(ecs_ctx* c, const cplx<R>* G2, R* out, const R* base, double* rowsq, int B, int mode,
                         cudaStream_t s) {
  RowFromBoxParams<R> p; p.G = G2; p.out = out; p.base = base; p.rowsq = rowsq; p.tw = (const cplx<R>*)c->tw;
  p.B = B; p.mode = mode;
  k_row_from_box<R, N, XT><<<B * (N / XT), XT * 32, smem_row_2f<R, N>(), s>>>(p);
}

template <typename R, int N>
void launch_col_rk4(ecs_ctx* c, int B, int stage, int produce, int diss, cudaStream_t s) {
  ColParams<R> p;
  p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.F = (cplx<R>*)c->F; p.A1 = (cplx<R>*)c->A1;
  p.K2 = (cplx<R>*)c->K2; p.OUT = (cplx<R>*)c->OUT; p.Etab = (const R*)c->Etab; p.ctl = c->ctl;
  p.fhat = (const cplx<R>*)c->fhat; p.tw = (const cplx<R>*)c->tw; p.nu = (R)c->nu; p.eta = (R)c->eta;
  p.B = B; p.stage = stage; p.produce = produce; p.diss = diss;
  const int cols = B * Geomc<N>::K;
  k_col_rk4<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
}

template <typename R, int N>
void launch_row_rhs(ecs_ctx* c, int B, R* phys, cudaStream_t s, const StepCtl* ctl = nullptr) {
  RowParams<R> p; p.G = (const cplx<R>*)c->G; p.H = (cplx<R>*)c->H; p.phys = phys; p.tw = (const cplx<R>*)c->tw;
  p.phys_bstride = 0; p.rec_index = 0; p.phys_stage = 0; p.ctl = ctl;
  p.b0x = (R)c->b0x; p.b0y = (R)c->b0y; p.B = B;
  k_row_rhs<R, N, XT><<<B * (N / XT), XT * 32, smem_row_rhs<R, N>(), s>>>(p);
}

template <typename R, int N>
void launch_col_rk43(ecs_ctx* c, int B, int stage, cudaStream_t s, cplx<R>* rec = nullptr, int cap = 0) {
  Col43Params<R> p;
  p.H = (const cplx<R>*)c->H; p.G = (cplx<R>*)c->G; p.S = (cplx<R>*)c->S43; p.ctl = c->ctl;
  p.fhat = (const cplx<R>*)c->fhat; p.tw = (const cplx<R>*)c->tw; p.rec = rec; p.cap = cap;
  p.nu = (R)c->nu; p.eta = (R)c->eta; p.B = B; p.stage = stage;
  const int cols = B * Geomc<N>::K;
  k_col_rk43<R, N><<<(cols + COLWARPS - 1) / COLWARPS, COLWARPS * 32, 0, s>>>(p);
}

template <typename R, int N>
void launch_row_err(ecs_ctx* c, int B, double atol, cudaStream_t s, double* rec_h = nullptr, int* rec_acc = nullptr,
                    int cap = 0) {
  RowErrParams<R> p; p.G = (const cplx<R>*)c->G; p.ctl = c->ctl; p.tw = (const cplx<R>*)c->tw; p.atol = atol;
  p.rec_h = rec_h; p.rec_acc = rec_acc; p.cap = cap; p.B = B;
  k_row_err<R, N, XT><<<B * (N / XT), XT * 32, smem_row_2f<R, N>(), s>>>(p);
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
    k_gather_box<R><<<grid1d(nbox), 256, 0, s>>>(fhat, (cplx<R>*)c->F, N, B);
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s);
    launch_row_rhs<R, N>(c, B, nullptr, s);
    launch_col_rk4<R, N>(c, B, COL_PLAIN, 0, diss, s);
    const long nfull = (long)B * 2 * N * (N / 2 + 1);
    k_scatter_box<R><<<grid1d(nfull), 256, 0, s>>>((const cplx<R>*)c->OUT, dfdt, N, B);
    return cuda_err(c, cudaGetLastError(), "state_vel");
  }

  // Lawson-RK4 over `steps` steps of the box state in c->F (ctl/Etab prepared).
  static int integrate_rk4(ecs_ctx* c, int B, long steps, cudaStream_t s) {
    if (steps <= 0) return ECS_OK;
    launch_col_rk4<R, N>(c, B, COL_START, 1, 0, s);
    for (long it = 0; it < steps; ++it) {
      for (int st = 1; st <= 4; ++st) {
        launch_row_rhs<R, N>(c, B, nullptr, s);
        launch_col_rk4<R, N>(c, B, st, (st == 4 && it == steps - 1) ? 0 : 1, 0, s);
      }
    }
    return cuda_err(c, cudaGetLastError(), "integrate_rk4");
  }

  static int rk4_setup(ecs_ctx* c, const double* T, int nc, int ms, int B, cudaStream_t s) {
    const long tot = (long)B * 2 * K * M;
    k_rk4_setup<R><<<grid1d(tot), 256, 0, s>>>(T, nc, ms, c->ctl, (R*)c->Etab, N, c->nu, c->eta, B);
    return cuda_err(c, cudaGetLastError(), "rk4_setup");
  }

  static int lawson_rk4(ecs_ctx* c, cplx<R>* fhat, double t, int steps, int B, cudaStream_t s) {
    k_fill<<<1, 256, 0, s>>>(c->Tbuf, t, B);
    int st = rk4_setup(c, c->Tbuf, 1, steps, B, s);
    if (st) return st;
    const long nbox = (long)B * 2 * K * M;
    k_gather_box<R><<<grid1d(nbox), 256, 0, s>>>(fhat, (cplx<R>*)c->F, N, B);
    st = integrate_rk4(c, B, steps, s);
    if (st) return st;
    const long nfull = (long)B * 2 * N * (N / 2 + 1);
    k_scatter_box<R><<<grid1d(nfull), 256, 0, s>>>((const cplx<R>*)c->F, fhat, N, B);
    return cuda_err(c, cudaGetLastError(), "lawson_rk4");
  }

  // Adaptive Lawson-RK4(3) of the box states in S43[b][S_X0] (timestepping.py:151-335).
  // Returns after all candidates completed or the attempt cap was reached.
  static int rk43_solve(ecs_ctx* c, const ecs_shoot_cfg* cfg, const double* T, int B, cudaStream_t s,
                        cplx<R>* rec = nullptr, double* rec_h = nullptr, int* rec_acc = nullptr, int cap = 0) {
    const long amax = (long)cfg->checkpoints * cfg->max_steps_per_checkpoint;
    if (amax <= 0) return set_err(c, ECS_ERR_INVALID, "checkpoints * max_steps_per_checkpoint must be > 0");
    k_rk43_setup<<<(B + 127) / 128, 128, 0, s>>>(T, cfg->h0, c->ctl, B);
    launch_col_rk43<R, N>(c, B, R43_START, s);
    launch_row_rhs<R, N>(c, B, nullptr, s, c->ctl);
    launch_col_rk43<R, N>(c, B, R43_INIT, s);
    for (long a = 0; a < amax; ++a) {
      launch_col_rk43<R, N>(c, B, R43_A, s, rec, cap);
      for (int st = R43_B; st <= R43_E; ++st) {
        launch_row_rhs<R, N>(c, B, nullptr, s, c->ctl);
        launch_col_rk43<R, N>(c, B, st, s, rec, cap);
      }
      launch_row_err<R, N>(c, B, cfg->atol, s, rec_h, rec_acc, cap);
      if ((a + 1) % 16 == 0 || a + 1 == amax) {
        k_count_done<<<1, 32, 0, s>>>(c->ctl, c->dcount, B);
        cudaError_t e = cudaMemcpyAsync(c->hcount, c->dcount, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return cuda_err(c, e, "rk43 completion check");
        if (*c->hcount == B) break;
      }
    }
    const long nbox = (long)B * 2 * K * M;
    k_rk43_resolve<R><<<grid1d(nbox), 256, 0, s>>>((cplx<R>*)c->S43, c->ctl, (cplx<R>*)c->F, N, B);
    return cuda_err(c, cudaGetLastError(), "rk43_solve");
  }

  // Forward shooting map + symmetries + residual (objective_RPO / loss_RPO).
  static int shoot(ecs_ctx* c, const ecs_shoot_cfg* cfg, const R* fields, const double* T, const double* sx,
                   R* out_fields, double* loss, ecs_info* info, int B, cudaStream_t s) {
    const bool rk43 = cfg->mode == ECS_MODE_LAWSON_RK43;
    if (cfg->mode != ECS_MODE_LAWSON_RK4 && !rk43)
      return set_err(c, ECS_ERR_BAD_MODE, "unknown integration mode");   // loss_functions.py:86-88
    int st;
    const long VEC = 2L * K * M;
    if (!rk43) {
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
    if (rk43) {   // modes outside the box are carried unchanged by the unmasked integrating factor
      launch_col_from_box<R, N>(c, (const cplx<R>*)c->V, (cplx<R>*)c->G, B, nullptr, 0, 0, 0, 0, s);
      launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, (R*)c->fields_tmp2, fields, nullptr, B, 1, s);
    }
    launch_col_from_box<R, N>(c, (const cplx<R>*)c->F, (cplx<R>*)c->G, B, sx, cfg->shift_reflect_ny, cfg->rot, 1, 0, s);
    launch_row_from_box<R, N>(c, (const cplx<R>*)c->G, out, fields, nullptr, B, 1, s);
    if (rk43) {
      const int odd = (cfg->shift_reflect_ny % 2 + 2) % 2 == 1;
      k_sub_sym_phys<R><<<grid1d((long)B * 2 * N * N), 256, 0, s>>>(out, (const R*)c->fields_tmp2, odd, cfg->rot, N, B);
    }
    if (loss) {
      k_rowsq<R><<<B * N, 32, 0, s>>>(out, c->rowsq, N);
      k_reduce_rows<<<(B + 127) / 128, 128, 0, s>>>(c->rowsq, loss, N, B, 1.0 / (2.0 * N * N));
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
};

}  // namespace ecs

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
#define ECS_DISPATCH(ctx, EXPR)                                                    \
  do {                                                                             \
    if ((ctx)->dtype == ECS_F64) {                                                 \
      switch ((ctx)->n) {                                                          \
        case 64:  { using R = double; constexpr int N = 64;  return EXPR; }        \
        case 128: { using R = double; constexpr int N = 128; return EXPR; }        \
        case 256: { using R = double; constexpr int N = 256; return EXPR; }        \
      }                                                                            \
    } else {                                                                       \
      switch ((ctx)->n) {                                                          \
        case 64:  { using R = float; constexpr int N = 64;  return EXPR; }         \
        case 128: { using R = float; constexpr int N = 128; return EXPR; }         \
        case 256: { using R = float; constexpr int N = 256; return EXPR; }         \
      }                                                                            \
    }                                                                              \
    return set_err(ctx, ECS_ERR_UNSUPPORTED, "unsupported n/dtype");               \
  } while (0)

#define ECS_CHECK_CTX(ctx, batch)                                                              \
  do {                                                                                         \
    if (!(ctx)) return ECS_ERR_INVALID;                                                        \
    if ((batch) < 1 || (batch) > (ctx)->max_batch)                                             \
      return set_err((ctx), ECS_ERR_INVALID, "batch must be in [1, max_batch]");              \
  } while (0)

static cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }

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
  c->G = dev_alloc(c, (size_t)B * 8 * Geomc<N>::K * N * cb, &st);
  c->H = dev_alloc(c, (size_t)B * 8 * Geomc<N>::K * N * cb, &st);
  c->fields_tmp = dev_alloc(c, (size_t)B * 2 * N * N * rb, &st);
  c->fields_tmp2 = dev_alloc(c, (size_t)B * 2 * N * N * rb, &st);
  c->S43 = dev_alloc(c, nbox * S_NSLOT * cb, &st);
  c->dcount = (int*)dev_alloc(c, sizeof(int), &st);
  c->ctl = (StepCtl*)dev_alloc(c, (size_t)B * sizeof(StepCtl), &st);
  c->rowsq = (double*)dev_alloc(c, (size_t)B * N * sizeof(double), &st);
  c->Tbuf = (double*)dev_alloc(c, (size_t)B * sizeof(double), &st);
  c->tw = dev_alloc(c, (N / 2) * cb, &st);
  c->fhat = dev_alloc(c, (size_t)Geomc<N>::K * Geomc<N>::M * cb, &st);
  if (st) return st;
  if (cudaMallocHost((void**)&c->hcount, sizeof(int)) != cudaSuccess) return set_err(c, ECS_ERR_OOM, "pinned alloc");
  // twiddles exp(-2 pi i k/N), k < N/2, from long double
  std::vector<cplx<R>> tw(N / 2);
  const long double twopi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < N / 2; ++k) {
    long double a = twopi * (long double)k / (long double)N;
    tw[k] = mk<R>((R)cosl(a), (R)(-sinl(a)));
  }
  cudaError_t e = cudaMemcpy(c->tw, tw.data(), tw.size() * cb, cudaMemcpyHostToDevice);
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

int ecs_ctx_create(int n, int dtype, const ecs_params* params, int max_batch, ecs_ctx** out) {
  if (!out || !params) return ECS_ERR_INVALID;
  *out = nullptr;
  if (!(n == 64 || n == 128 || n == 256)) return ECS_ERR_UNSUPPORTED;
  if (!(dtype == ECS_F64 || dtype == ECS_F32)) return ECS_ERR_UNSUPPORTED;
  if (max_batch < 1) return ECS_ERR_INVALID;
  ecs_ctx* c = new ecs_ctx();
  c->n = n; c->dtype = dtype; c->max_batch = max_batch; c->g = make_geom(n);
  c->nu = params->nu; c->eta = params->eta; c->b0x = params->b0x; c->b0y = params->b0y;
  int st;
  {
    auto run = [&]() -> int { ECS_DISPATCH(c, (ctx_init<R, N>(c, params))); };
    st = run();
  }
  if (st != ECS_OK) {
    fprintf(stderr, "ecs_ctx_create: %s\n", c->err.c_str());
    ecs_ctx_destroy(c);
    return st;
  }
  *out = c;
  return ECS_OK;
}

int ecs_ctx_destroy(ecs_ctx* ctx) {
  if (!ctx) return ECS_OK;
  cudaDeviceSynchronize();
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->hcount) cudaFreeHost(ctx->hcount);
  delete ctx;
  return ECS_OK;
}

int ecs_to_box(ecs_ctx* ctx, const void* fields, void* box, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!fields || !box) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  ECS_DISPATCH(ctx, (Impl<R, N>::to_box(ctx, (const R*)fields, (cplx<R>*)box, batch, as_stream(stream))));
}

int ecs_from_box(ecs_ctx* ctx, const void* box, void* fields, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!fields || !box) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  ECS_DISPATCH(ctx, (Impl<R, N>::from_box(ctx, (const cplx<R>*)box, (R*)fields, batch, as_stream(stream))));
}

int ecs_dealias(ecs_ctx* ctx, const void* fields, void* out, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!fields || !out) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  ECS_DISPATCH(ctx, (Impl<R, N>::dealias(ctx, (const R*)fields, (R*)out, batch, as_stream(stream))));
}

int ecs_state_vel(ecs_ctx* ctx, const void* f_hat, void* dfdt_hat, int batch, int include_dissipation, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!f_hat || !dfdt_hat) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  ECS_DISPATCH(ctx, (Impl<R, N>::state_vel(ctx, (const cplx<R>*)f_hat, (cplx<R>*)dfdt_hat, batch,
                                           include_dissipation, as_stream(stream))));
}

int ecs_lawson_rk4(ecs_ctx* ctx, void* f_hat, double t, int steps, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!f_hat) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  if (steps < 1) return set_err(ctx, ECS_ERR_INVALID, "steps must be >= 1");
  ECS_DISPATCH(ctx, (Impl<R, N>::lawson_rk4(ctx, (cplx<R>*)f_hat, t, steps, batch, as_stream(stream))));
}

int ecs_objective(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T, const double* sx,
                  void* out_fields, double* out_T, double* out_sx, ecs_info* info, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfg || !fields || !T || !sx || !out_fields) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  cudaStream_t s = as_stream(stream);
  // phase conditions pt - stop_gradient(pt) are exactly 0 in value (loss_functions.py:128-129)
  if (out_T) { cudaError_t e = cudaMemsetAsync(out_T, 0, sizeof(double) * batch, s); if (e) return cuda_err(ctx, e, "out_T"); }
  if (out_sx) { cudaError_t e = cudaMemsetAsync(out_sx, 0, sizeof(double) * batch, s); if (e) return cuda_err(ctx, e, "out_sx"); }
  ECS_DISPATCH(ctx, (Impl<R, N>::shoot(ctx, cfg, (const R*)fields, T, sx, (R*)out_fields, nullptr, info, batch, s)));
}

int ecs_loss(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T, const double* sx,
             double* loss, ecs_info* info, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfg || !fields || !T || !sx || !loss) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  ECS_DISPATCH(ctx, (Impl<R, N>::shoot(ctx, cfg, (const R*)fields, T, sx, nullptr, loss, info, batch, as_stream(stream))));
}
