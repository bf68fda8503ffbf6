// Instantiation of the F32 n=64 kernels and host operations.
#include "impl.cuh"

const ecs::ImplTable* ecs::impl_table_f32_64() {
  static const ImplTable t = make_table<float, 64>();
  return &t;
}
