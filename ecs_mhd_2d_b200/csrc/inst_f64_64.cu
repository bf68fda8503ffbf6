// Instantiation of the F64 n=64 kernels and host operations.
#include "impl.cuh"

const ecs::ImplTable* ecs::impl_table_f64_64() {
  static const ImplTable t = make_table<double, 64>();
  return &t;
}
