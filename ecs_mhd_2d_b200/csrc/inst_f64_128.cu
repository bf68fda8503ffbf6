// Instantiation of the F64 n=128 kernels and host operations.
#include "impl.cuh"

const ecs::ImplTable* ecs::impl_table_f64_128() {
  static const ImplTable t = make_table<double, 128>();
  return &t;
}
