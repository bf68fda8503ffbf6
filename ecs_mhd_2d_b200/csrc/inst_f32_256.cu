// Instantiation of the F32 n=256 kernels and host operations.
#include "impl.cuh"

const ecs::ImplTable* ecs::impl_table_f32_256() {
  static const ImplTable t = make_table<float, 256>();
  return &t;
}
