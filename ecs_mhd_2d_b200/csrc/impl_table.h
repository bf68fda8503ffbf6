// Per-(dtype, n) function table of the C-ABI operations (filled in inst_*.cu).
#pragma once

#include <cuda_runtime.h>

#include "../../include/ecs_mhd.h"

struct ecs_ctx;

namespace ecs {

struct ImplTable {
  int (*init)(ecs_ctx*, const ecs_params*);
  int (*to_box)(ecs_ctx*, const void*, void*, int, cudaStream_t);
  int (*from_box)(ecs_ctx*, const void*, void*, int, cudaStream_t);
  int (*dealias)(ecs_ctx*, const void*, void*, int, cudaStream_t);
  int (*state_vel)(ecs_ctx*, const void*, void*, int, int, cudaStream_t);
  int (*lawson_rk4)(ecs_ctx*, void*, double, int, int, cudaStream_t);
  int (*shoot)(ecs_ctx*, const ecs_shoot_cfg*, const void*, const double*, const double*, void*, double*, ecs_info*,
               int, cudaStream_t);
  int (*linearize)(ecs_ctx*, const ecs_shoot_cfg*, const void*, const double*, const double*, void*, ecs_info*,
                   cudaStream_t);
  int (*jvp)(ecs_ctx*, const void*, const double*, const double*, void*, double*, double*, int, cudaStream_t);
  int (*integrate)(ecs_ctx*, int, void*, double, int, int, cudaStream_t);
  int (*recurrence)(ecs_ctx*, const void*, int, double*, cudaStream_t);
  int (*linearize_jvp)(ecs_ctx*, const ecs_shoot_cfg*, const void*, const double*, const double*, void*, ecs_info*,
                       const void*, const double*, const double*, void*, double*, double*, int, cudaStream_t);
  int (*vjp)(ecs_ctx*, const void*, const double*, const double*, void*, double*, double*, int, cudaStream_t);
  int (*bench_kernel)(ecs_ctx*, int, int, int, float*, double*, cudaStream_t);
  int (*jvp_multi)(ecs_ctx*, const ecs_shoot_cfg*, const void*, const double*, const double*, void*, const void*,
                   const double*, const double*, void*, double*, double*, int, cudaStream_t);
  int (*loss_grad_multi)(ecs_ctx*, const ecs_shoot_cfg*, const void*, const double*, const double*, double*, void*,
                         double*, double*, int, cudaStream_t);
  int (*pool_reset)(ecs_ctx*, cudaStream_t);
  int (*pool_admit)(ecs_ctx*, int, const ecs_shoot_cfg*, const void*, double, double, cudaStream_t);
  int (*pool_advance)(ecs_ctx*, int, cudaStream_t);
  int (*pool_retire)(ecs_ctx*, int, void*, double*, cudaStream_t);
};

const ImplTable* impl_table_f64_64();
const ImplTable* impl_table_f64_128();
const ImplTable* impl_table_f64_256();
const ImplTable* impl_table_f32_64();
const ImplTable* impl_table_f32_128();
const ImplTable* impl_table_f32_256();

inline const ImplTable* impl_table(int dtype, int n) {
  if (dtype == ECS_F64) {
    if (n == 64) return impl_table_f64_64();
    if (n == 128) return impl_table_f64_128();
    if (n == 256) return impl_table_f64_256();
  } else if (dtype == ECS_F32) {
    if (n == 64) return impl_table_f32_64();
    if (n == 128) return impl_table_f32_128();
    if (n == 256) return impl_table_f32_256();
  }
  return nullptr;
}

}  // namespace ecs
