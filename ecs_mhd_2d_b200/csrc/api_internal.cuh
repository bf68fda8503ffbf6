// Host-side context shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "common.cuh"

struct ecs_ctx {
  int n = 0, dtype = 0, max_batch = 0;
  ecs::Geom g{};
  double nu = 0, eta = 0, b0x = 0, b0y = 0;
  // tables
  void* tw = nullptr;      // [N/2] twiddles
  void* fhat = nullptr;    // [K][M] forcing box spectrum (omega)
  // workspace, sized for max_batch
  void* F = nullptr;       // box state / accumulator
  void* A1 = nullptr;      // e*k1
  void* K2 = nullptr;      // k2
  void* OUT = nullptr;     // state_vel output
  void* V = nullptr;       // scratch box vector
  void* Etab = nullptr;    // exp(h/2 L) mask
  void* G = nullptr;       // [B][8][K][N]
  void* H = nullptr;       // [B][8][K][N]
  void* fields_tmp = nullptr;  // [B][2][N][N]
  void* fields_tmp2 = nullptr; // [B][2][N][N]
  void* S43 = nullptr;         // [B][S_NSLOT][2][K][M] adaptive stepper slots
  int* dcount = nullptr;       // device completion counter
  int* hcount = nullptr;       // pinned host mirror
  ecs::StepCtl* ctl = nullptr;
  double* rowsq = nullptr;
  double* Tbuf = nullptr;
  std::vector<void*> allocs;
  std::string err;
};

namespace ecs {

template <int N> struct Geomc {
  static constexpr int kmax = (N - 1) / 3;
  static constexpr int K = kmax + 1;
  static constexpr int M = 2 * kmax + 1;
};

int set_err(ecs_ctx* c, int code, const std::string& msg);
int cuda_err(ecs_ctx* c, cudaError_t e, const char* where);
void* dev_alloc(ecs_ctx* c, size_t bytes, int* st);

static __global__ void k_fill(double* p, double v, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}

}  // namespace ecs
