// Instantiation of the F32 n=128 kernels and host operations.
#include "impl.cuh"

const ecs::ImplTable* ecs::impl_table_f32_128() {
  static const ImplTable t = make_table<float, 128>();
  return &t;
}
