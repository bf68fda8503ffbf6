// Instantiation of the F64 n=256 kernels and host operations.
#include "impl.cuh"

const ecs::ImplTable* ecs::impl_table_f64_256() {
  static const ImplTable t = make_table<double, 256>();
  return &t;
}
