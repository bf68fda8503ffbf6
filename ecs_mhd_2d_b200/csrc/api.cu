// C ABI of the ECS-MHD-2D B200 hot path: context, workspace, dispatch and the
// host-side orchestration of the kernels in kernels.cuh.
#include "../../include/ecs_mhd.h"
#include "api_internal.cuh"
#include "impl_table.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>

using namespace ecs;

const char* ecs_version(void) { return "ecs_mhd_2d_b200 0.1 (sm_100a)"; }

const char* ecs_last_error(const ecs_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int ecs_box_dims(const ecs_ctx* ctx, int* K, int* M) {
  if (!ctx || !K || !M) return ECS_ERR_INVALID;
  *K = ctx->g.K; *M = ctx->g.M;
  return ECS_OK;
}

namespace ecs {

std::mutex& capture_mutex() {
  static std::mutex m;
  return m;
}

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

int grow(ecs_ctx* c, void** p, size_t* have, size_t need) {
  if (*have >= need && *p) return ECS_OK;
  if (*p) { cudaFree(*p); *p = nullptr; *have = 0; }
  cudaError_t e = cudaMalloc(p, need < 256 ? 256 : need);
  if (e != cudaSuccess) { *p = nullptr; return set_err(c, ECS_ERR_OOM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e)); }
  *have = need;
  return ECS_OK;
}

}  // namespace ecs

// ---------------------------------------------------------------------------
// dispatch
// ---------------------------------------------------------------------------
// Function table for the context's (dtype, n).
static const ecs::ImplTable* table_of(const ecs_ctx* c) { return ecs::impl_table(c->dtype, c->n); }

#define ECS_CHECK_CTX(ctx, batch)                                                              \
  do {                                                                                         \
    if (!(ctx)) return ECS_ERR_INVALID;                                                        \
    if ((batch) < 1 || (batch) > (ctx)->max_batch)                                             \
      return set_err((ctx), ECS_ERR_INVALID, "batch must be in [1, max_batch]");              \
  } while (0)

static cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }


static int ctx_destroy_locked(ecs_ctx* ctx);

int ecs_ctx_create(int n, int dtype, const ecs_params* params, int max_batch, ecs_ctx** out) {
  if (!out || !params) return ECS_ERR_INVALID;
  *out = nullptr;
  if (!(n == 64 || n == 128 || n == 256)) return ECS_ERR_UNSUPPORTED;
  if (!(dtype == ECS_F64 || dtype == ECS_F32)) return ECS_ERR_UNSUPPORTED;
  if (max_batch < 1) return ECS_ERR_INVALID;
  std::lock_guard<std::mutex> capture_guard(ecs::capture_mutex());   // set-up synchronises the device
  ecs_ctx* c = new ecs_ctx();
  c->n = n; c->dtype = dtype; c->max_batch = max_batch; c->g = make_geom(n);
  c->nu = params->nu; c->eta = params->eta; c->b0x = params->b0x; c->b0y = params->b0y;
  if (const char* v = getenv("ECS_PDL")) c->pdl = atoi(v) != 0 ? 1 : 0;
  if (const char* v = getenv("ECS_TGROUPS")) c->tgroups = std::max(1, std::min(ecs_ctx::MAXG, atoi(v)));
  if (const char* v = getenv("ECS_ROWTAN_XT")) c->rowtan_xt = atoi(v) == 4 ? 4 : 8;
  if (const char* v = getenv("ECS_PDL_MINB")) c->pdl_minb = std::max(1, atoi(v));
  if (const char* v = getenv("ECS_CHAIN_MAXB")) c->chain_maxb = std::max(0, atoi(v));
  if (const char* v = getenv("ECS_RK4CHAIN_MAXB")) c->rk4chain_maxb = std::max(0, atoi(v));
  if (const char* v = getenv("ECS_CHAIN_DSMEM")) c->chain_dsm = atoi(v) != 0 ? 1 : 0;
  if (const char* v = getenv("ECS_CHAIN_DSLOTS")) c->chain_dsh = atoi(v) != 0 ? 1 : 0;
  if (const char* v = getenv("ECS_CHAIN_WARPS")) c->chain_w = atoi(v) == 16 ? 16 : atoi(v) == 8 ? 8 : 0;
  if (const char* v = getenv("ECS_CHAIN_MINB")) c->chain_minb = std::max(1, atoi(v));
  if (const char* v = getenv("ECS_RK4CHAIN_MINB")) c->rk4chain_minb = std::max(1, atoi(v));
  if (const char* v = getenv("ECS_RK43CHAIN_MINB")) c->rk43chain_minb = std::max(1, atoi(v));
  if (const char* v = getenv("ECS_RK43CHAIN_MAXB")) c->rk43chain_maxb = std::max(0, atoi(v));
  if (const char* v = getenv("ECS_REGEN_ITEMS")) c->regen_items = atoi(v) > 0 ? std::max(8, atoi(v)) : 0;
  int st;
  const ecs::ImplTable* t = ecs::impl_table(dtype, n);
  st = t ? t->init(c, params) : ECS_ERR_UNSUPPORTED;
  if (st != ECS_OK) {
    fprintf(stderr, "ecs_ctx_create: %s\n", c->err.c_str());
    ctx_destroy_locked(c);
    return st;
  }
  *out = c;
  return ECS_OK;
}

static int ctx_destroy_locked(ecs_ctx* ctx) {
  if (!ctx) return ECS_OK;
  cudaDeviceSynchronize();
  for (void* p : ctx->allocs) cudaFree(p);
  if (ctx->hcount) cudaFreeHost(ctx->hcount);
  if (ctx->g43.exec) cudaGraphExecDestroy(ctx->g43.exec);
  if (ctx->g4.exec) cudaGraphExecDestroy(ctx->g4.exec);
  for (auto& g : ctx->gfx) if (g.exec) cudaGraphExecDestroy(g.exec);
  if (ctx->fxphys) cudaFree(ctx->fxphys);
  if (ctx->gpool.exec) cudaGraphExecDestroy(ctx->gpool.exec);
  if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
  if (ctx->pstream) cudaStreamDestroy(ctx->pstream);
  for (cudaEvent_t e : ctx->pev) if (e) cudaEventDestroy(e);
  for (int g = 0; g < ecs_ctx::MAXG; ++g) {
    if (ctx->tstream[g]) cudaStreamDestroy(ctx->tstream[g]);
    for (cudaEvent_t e : ctx->tjoin[g]) if (e) cudaEventDestroy(e);
  }
  if (ctx->tfork) cudaEventDestroy(ctx->tfork);
  for (cudaEvent_t e : ctx->kt.ev) cudaEventDestroy(e);
  if (ctx->mj.g.exec) cudaGraphExecDestroy(ctx->mj.g.exec);
  for (void* p : {ctx->mj.ckpt, ctx->mj.grec, ctx->mj.gphys, ctx->mj.res}) if (p) cudaFree(p);
  if (ctx->Gp) cudaFree(ctx->Gp);
  if (ctx->Gx) cudaFree(ctx->Gx);
  if (ctx->Hp) cudaFree(ctx->Hp);
  if (ctx->hctl) cudaFreeHost(ctx->hctl);
  if (ctx->hchunk_acc) cudaFreeHost(ctx->hchunk_acc);
  if (ctx->hchunk_h) cudaFreeHost(ctx->hchunk_h);
  if (ctx->hitems) cudaFreeHost(ctx->hitems);
  if (ctx->lin.rec) cudaFree(ctx->lin.rec);
  if (ctx->lin.ckpt) cudaFree(ctx->lin.ckpt);
  if (ctx->lin.rec2) cudaFree(ctx->lin.rec2);
  if (ctx->lin.rec_h) cudaFree(ctx->lin.rec_h);
  if (ctx->lin.rec_acc) cudaFree(ctx->lin.rec_acc);
  if (ctx->D) cudaFree(ctx->D);
  if (ctx->chain_ops) cudaFree(ctx->chain_ops);
  if (ctx->Greg) cudaFree(ctx->Greg);
  if (ctx->Phys) cudaFree(ctx->Phys);
  if (ctx->items) cudaFree(ctx->items);
  if (ctx->hacc) cudaFree(ctx->hacc);
  delete ctx;
  return ECS_OK;
}

int ecs_ctx_destroy(ecs_ctx* ctx) {
  std::lock_guard<std::mutex> capture_guard(ecs::capture_mutex());   // synchronises the device
  return ctx_destroy_locked(ctx);
}

int ecs_to_box(ecs_ctx* ctx, const void* fields, void* box, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!fields || !box) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->to_box(ctx, fields, box, batch, as_stream(stream));
}

int ecs_from_box(ecs_ctx* ctx, const void* box, void* fields, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!fields || !box) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->from_box(ctx, box, fields, batch, as_stream(stream));
}

int ecs_dealias(ecs_ctx* ctx, const void* fields, void* out, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!fields || !out) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->dealias(ctx, fields, out, batch, as_stream(stream));
}

int ecs_state_vel(ecs_ctx* ctx, const void* f_hat, void* dfdt_hat, int batch, int include_dissipation, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!f_hat || !dfdt_hat) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->state_vel(ctx, f_hat, dfdt_hat, batch,
                                           include_dissipation, as_stream(stream));
}

int ecs_lawson_rk4(ecs_ctx* ctx, void* f_hat, double t, int steps, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!f_hat) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  if (steps < 1) return set_err(ctx, ECS_ERR_INVALID, "steps must be >= 1");
  return table_of(ctx)->lawson_rk4(ctx, f_hat, t, steps, batch, as_stream(stream));
}

int ecs_integrate(ecs_ctx* ctx, int mode, void* f_hat, double t, int steps, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!f_hat) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  if (steps < 1) return set_err(ctx, ECS_ERR_INVALID, "steps must be >= 1");
  return table_of(ctx)->integrate(ctx, mode, f_hat, t, steps, batch, as_stream(stream));
}

int ecs_recurrence(ecs_ctx* ctx, const void* fs, int snapshots, double* dist, void* stream) {
  if (!ctx) return ECS_ERR_INVALID;
  if (!fs || !dist || snapshots < 1 || snapshots > 65535) return set_err(ctx, ECS_ERR_INVALID, "bad arguments");
  return table_of(ctx)->recurrence(ctx, fs, snapshots, dist, as_stream(stream));
}

int ecs_objective(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T, const double* sx,
                  void* out_fields, double* out_T, double* out_sx, ecs_info* info, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfg || !fields || !T || !sx || !out_fields) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  cudaStream_t s = as_stream(stream);
  // phase conditions pt - stop_gradient(pt) are exactly 0 in value (loss_functions.py:128-129)
  if (out_T) { cudaError_t e = cudaMemsetAsync(out_T, 0, sizeof(double) * batch, s); if (e) return cuda_err(ctx, e, "out_T"); }
  if (out_sx) { cudaError_t e = cudaMemsetAsync(out_sx, 0, sizeof(double) * batch, s); if (e) return cuda_err(ctx, e, "out_sx"); }
  return table_of(ctx)->shoot(ctx, cfg, fields, T, sx, out_fields, nullptr, info, batch, s);
}

int ecs_loss(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T, const double* sx,
             double* loss, ecs_info* info, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfg || !fields || !T || !sx || !loss) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->shoot(ctx, cfg, fields, T, sx, nullptr, loss, info, batch, as_stream(stream));
}

int ecs_linearize(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T, const double* sx,
                  void* out_fields, ecs_info* info, void* stream) {
  ECS_CHECK_CTX(ctx, 1);
  if (!cfg || !fields || !T || !sx) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->linearize(ctx, cfg, fields, T, sx, out_fields, info, as_stream(stream));
}

int ecs_jvp(ecs_ctx* ctx, const void* dfields, const double* dT, const double* dsx, void* out_dfields,
            double* out_dT, double* out_dsx, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!dfields || !dT || !dsx || !out_dfields || !out_dT || !out_dsx) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->jvp(ctx, dfields, dT, dsx, out_dfields, out_dT, out_dsx, batch,
                                     as_stream(stream));
}

int ecs_linearize_jvp(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T, const double* sx,
                      void* out_fields, ecs_info* info, const void* dfields, const double* dT, const double* dsx,
                      void* out_dfields, double* out_dT, double* out_dsx, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfg || !fields || !T || !sx || !dfields || !dT || !dsx || !out_dfields || !out_dT || !out_dsx)
    return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->linearize_jvp(ctx, cfg, fields, T, sx, out_fields, info, dfields, dT, dsx, out_dfields, out_dT,
                                      out_dsx, batch, as_stream(stream));
}

int ecs_vjp(ecs_ctx* ctx, const void* c_fields, const double* c_T, const double* c_sx, void* g_fields, double* g_T,
            double* g_sx, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!c_fields || !c_T || !c_sx || !g_fields || !g_T || !g_sx) return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->vjp(ctx, c_fields, c_T, c_sx, g_fields, g_T, g_sx, batch,
                                     as_stream(stream));
}

long long ecs_launch_count(const ecs_ctx* ctx) { return ctx ? ctx->launches : -1; }

int ecs_bench_kernel(ecs_ctx* ctx, int which, int batch, int iters, float* ms, double* bytes, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!ms || !bytes || iters < 1 || which < 0 || which > 1) return set_err(ctx, ECS_ERR_INVALID, "bad arguments");
  return table_of(ctx)->bench_kernel(ctx, which, batch, iters, ms, bytes, as_stream(stream));
}

int ecs_jvp_multi(ecs_ctx* ctx, const ecs_shoot_cfg* cfgs, const void* fields, const double* T, const double* sx,
                  void* out_fields, const void* dfields, const double* dT, const double* dsx, void* out_dfields,
                  double* out_dT, double* out_dsx, int batch, void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfgs || !fields || !T || !sx || !dfields || !dT || !dsx || !out_dfields || !out_dT || !out_dsx)
    return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->jvp_multi(ctx, cfgs, fields, T, sx, out_fields, dfields, dT, dsx, out_dfields, out_dT, out_dsx,
                                  batch, as_stream(stream));
}

int ecs_loss_grad_multi(ecs_ctx* ctx, const ecs_shoot_cfg* cfgs, const void* fields, const double* T,
                        const double* sx, double* loss, void* g_fields, double* g_T, double* g_sx, int batch,
                        void* stream) {
  ECS_CHECK_CTX(ctx, batch);
  if (!cfgs || !fields || !T || !sx || !loss || !g_fields || !g_T || !g_sx)
    return set_err(ctx, ECS_ERR_INVALID, "null pointer");
  return table_of(ctx)->loss_grad_multi(ctx, cfgs, fields, T, sx, loss, g_fields, g_T, g_sx, batch, as_stream(stream));
}

namespace ecs {
static cudaEvent_t kt_event(ecs_ctx* c) {
  auto& k = c->kt;
  if (k.used == k.ev.size()) {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) { k.on = 0; return nullptr; }
    k.ev.push_back(e);
  }
  return k.ev[k.used++];
}

void kt_begin(ecs_ctx* c, cudaStream_t s) {
  if (!c->kt.on) return;
  cudaEvent_t e = kt_event(c);
  if (e) cudaEventRecord(e, s);
}

void kt_end(ecs_ctx* c, int kind, int batch, cudaStream_t s) {
  if (!c->kt.on) return;
  cudaEvent_t e = kt_event(c);
  if (!e) return;
  cudaEventRecord(e, s);
  c->kt.kind.push_back(kind);
  c->kt.batch = batch;
}
}  // namespace ecs

int ecs_kernel_timing(ecs_ctx* ctx, int enable, double* row_ms, int* row_n, double* col_ms, int* col_n,
                      int* group_batch) {
  if (!ctx) return ECS_ERR_INVALID;
  auto& k = ctx->kt;
  if (enable) {
    k.on = 1; k.used = 0; k.batch = 0; k.kind.clear();
    return ECS_OK;
  }
  k.on = 0;
  double sum[2] = {0, 0};
  int cnt[2] = {0, 0};
  for (size_t i = 0; i < k.kind.size(); ++i) {
    if (2 * i + 1 >= k.used) break;
    float ms = 0;
    cudaError_t e = cudaEventSynchronize(k.ev[2 * i + 1]);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, k.ev[2 * i], k.ev[2 * i + 1]);
    if (e != cudaSuccess) return set_err(ctx, ECS_ERR_CUDA, cudaGetErrorString(e));
    sum[k.kind[i]] += ms;
    ++cnt[k.kind[i]];
  }
  if (row_ms) *row_ms = cnt[0] ? sum[0] / cnt[0] : 0.0;
  if (row_n) *row_n = cnt[0];
  if (col_ms) *col_ms = cnt[1] ? sum[1] / cnt[1] : 0.0;
  if (col_n) *col_n = cnt[1];
  if (group_batch) *group_batch = k.batch;
  k.used = 0; k.kind.clear();
  return ECS_OK;
}

int ecs_pool_reset(ecs_ctx* ctx, void* stream) {
  if (!ctx) return ECS_ERR_INVALID;
  return table_of(ctx)->pool_reset(ctx, as_stream(stream));
}

int ecs_pool_admit(ecs_ctx* ctx, int slot, const ecs_shoot_cfg* cfg, const void* fields, double T, double sx,
                   void* stream) {
  if (!ctx || !cfg || !fields) return ECS_ERR_INVALID;
  if (slot < 0 || slot >= ctx->max_batch) return set_err(ctx, ECS_ERR_INVALID, "slot out of range");
  return table_of(ctx)->pool_admit(ctx, slot, cfg, fields, T, sx, as_stream(stream));
}

int ecs_pool_advance(ecs_ctx* ctx, int nsteps, void* stream) {
  if (!ctx || nsteps < 1) return ECS_ERR_INVALID;
  return table_of(ctx)->pool_advance(ctx, nsteps, as_stream(stream));
}

int ecs_pool_poll(ecs_ctx* ctx, int* done, int* steps_done, void* stream) {
  if (!ctx || !done) return ECS_ERR_INVALID;
  std::vector<ecs::StepCtl> h(ctx->max_batch);
  cudaError_t e = cudaMemcpyAsync(h.data(), ctx->ctl, sizeof(ecs::StepCtl) * ctx->max_batch, cudaMemcpyDeviceToHost,
                                  as_stream(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
  if (e != cudaSuccess) return set_err(ctx, ECS_ERR_CUDA, cudaGetErrorString(e));
  for (int b = 0; b < ctx->max_batch; ++b) {
    const bool active = b < (int)ctx->pool.size() && ctx->pool[b].active;
    done[b] = active ? h[b].done : 0;
    if (steps_done) steps_done[b] = active ? h[b].steps_done : 0;
  }
  return ECS_OK;
}

int ecs_pool_retire(ecs_ctx* ctx, int slot, void* out_fields, double* loss, void* stream) {
  if (!ctx) return ECS_ERR_INVALID;
  if (slot < 0 || slot >= (int)ctx->pool.size() || !ctx->pool[slot].active)
    return set_err(ctx, ECS_ERR_INVALID, "slot not active");
  return table_of(ctx)->pool_retire(ctx, slot, out_fields, loss, as_stream(stream));
}
