// state_vel without any device allocation, for callers that cannot allocate.
//
// Who needs it: a host process whose device memory is owned by another
// allocator.  The reference runs under JAX, whose XLA client preallocates most
// of the GPU's memory at start-up and hands buffers to custom calls; a library
// that calls cudaMalloc inside such a process can fail (the memory is already
// taken) or fragment the pool.  Real-time or embedded callers that forbid
// allocation after start-up are in the same position.  This entry point runs
// the same fused state_vel kernels as ecs_state_vel but takes every byte of its
// scratch from one file-scope device array of fixed size.
//
// Limits: FP64, n in {64, 128}, batch <= 4; the array is ~3.8 MB and stays
// resident on every GPU that loads the library until the process exits.
// Calls share the array: two calls that overlap on the GPU (different streams,
// or different host threads on one device) race and corrupt each other.
// The first call on each device performs a one-time set-up (symbol address
// lookup, twiddle upload, kernel attributes) with synchronous CUDA calls, so
// that first call should come before any stream capture.  The device address
// found then is kept for the life of the process, per device ordinal: the entry
// point assumes the CUDA runtime's primary context of that device and no
// cudaDeviceReset afterwards (a reset frees the module memory behind it).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "../../include/ecs_mhd.h"
#include "api_internal.cuh"
#include "kernels.cuh"

namespace {

using namespace ecs;

constexpr int NA_MAX_N = 128;
constexpr int NA_MAX_BATCH = 4;
constexpr int NA_XT = 8;
constexpr size_t NA_K = (NA_MAX_N - 1) / 3 + 1;
constexpr size_t NA_M = 2 * ((NA_MAX_N - 1) / 3) + 1;
constexpr size_t CB = sizeof(double2);
constexpr size_t al(size_t x) { return (x + 255) / 256 * 256; }

// Byte layout of the static scratch (sized for n = 128, batch = 4).
constexpr size_t OFF_TW64 = 0;                                                   // twiddle image, n = 64
constexpr size_t OFF_TW128 = al(OFF_TW64 + tw_smem(64) * CB);                    // twiddle image, n = 128
constexpr size_t OFF_CTL = al(OFF_TW128 + tw_smem(128) * CB);                    // step controls (zeroed)
constexpr size_t OFF_FIELDS = al(OFF_CTL + NA_MAX_BATCH * sizeof(StepCtl));      // [forcing; 0] real [2][n][n]
constexpr size_t OFF_FBOX = al(OFF_FIELDS + 2 * NA_MAX_N * NA_MAX_N * sizeof(double));   // forcing box [2][K][M]
constexpr size_t OFF_F = al(OFF_FBOX + 2 * NA_K * NA_M * CB);                    // input box [B][2][K][M]
constexpr size_t OFF_OUT = al(OFF_F + NA_MAX_BATCH * 2 * NA_K * NA_M * CB);      // output box
constexpr size_t OFF_G = al(OFF_OUT + NA_MAX_BATCH * 2 * NA_K * NA_M * CB);      // [B][NG][K][n]
constexpr size_t OFF_H = al(OFF_G + NA_MAX_BATCH * NG * NA_K * NA_MAX_N * CB);   // [B][NH][K][n]
constexpr size_t NA_BYTES = al(OFF_H + NA_MAX_BATCH * NH * NA_K * NA_MAX_N * CB);

unsigned char* g_base[128] = {};   // device address of the scratch array, per device ordinal

}  // namespace

// The scratch: one fixed-size array per device, shared by every call.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_BYTES];

namespace {

template <int N>
int na_setup_twiddles(unsigned char* base, size_t off) {
  std::vector<double2> tw(N / 2);
  const long double twopi = 6.283185307179586476925286766559005768L;
  for (int k = 0; k < N / 2; ++k) {
    const long double a = twopi * (long double)k / (long double)N;
    tw[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
  }
  std::vector<double2> img(tw_smem(N));
  twiddle_image<double2, N>(tw.data(), img.data());
  return cudaMemcpy(base + off, img.data(), img.size() * CB, cudaMemcpyHostToDevice) == cudaSuccess ? ECS_OK
                                                                                                  : ECS_ERR_CUDA;
}

template <int N> size_t na_smem_rhs() { return (fft_smem(N, NA_XT) + (NG + NH) * ((N - 1) / 3 + 1) * (NA_XT + 1)) * CB; }
template <int N> size_t na_smem_2f() { return (fft_smem(N, NA_XT) + 2 * ((N - 1) / 3 + 1) * (NA_XT + 1)) * CB; }

// One-time set-up on the current device (synchronous).  It holds the mutex that
// context set-up and every graph capture of this library take, so its
// legacy-stream copies never land inside another thread's capture.
int na_setup(unsigned char** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return ECS_ERR_CUDA;
  std::lock_guard<std::mutex> lock(ecs::capture_mutex());
  if (!g_base[dev]) {
    void* p = nullptr;
    // In host code g_noalloc_scratch names a host-side stand-in; the kernels
    // need the device address, which only cudaGetSymbolAddress gives.
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return ECS_ERR_CUDA;
    unsigned char* base = static_cast<unsigned char*>(p);
    if (na_setup_twiddles<64>(base, OFF_TW64) || na_setup_twiddles<128>(base, OFF_TW128)) return ECS_ERR_CUDA;
    cudaError_t e = cudaFuncSetAttribute(k_row_rhs<double, 128, NA_XT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)na_smem_rhs<128>());
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_row_rhs<double, 64, NA_XT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)na_smem_rhs<64>());
    if (e != cudaSuccess) return ECS_ERR_CUDA;
    g_base[dev] = base;
  }
  *out = g_base[dev];
  return ECS_OK;
}

template <int N>
int na_state_vel(unsigned char* base, double nu, double eta, double b0x, double b0y, const double* forcing,
                 const double2* f_hat, double2* dfdt, int B, int diss, cudaStream_t s) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  const double2* tw = reinterpret_cast<const double2*>(base + (N == 64 ? OFF_TW64 : OFF_TW128));
  double* fields = reinterpret_cast<double*>(base + OFF_FIELDS);
  double2* fbox = reinterpret_cast<double2*>(base + OFF_FBOX);
  double2* F = reinterpret_cast<double2*>(base + OFF_F);
  double2* OUT = reinterpret_cast<double2*>(base + OFF_OUT);
  double2* G = reinterpret_cast<double2*>(base + OFF_G);
  double2* H = reinterpret_cast<double2*>(base + OFF_H);
  StepCtl* ctl = reinterpret_cast<StepCtl*>(base + OFF_CTL);
  // the array keeps the previous call's contents: clear what must start at zero
  cudaError_t e = cudaMemsetAsync(ctl, 0, NA_MAX_BATCH * sizeof(StepCtl), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(fields, forcing, (size_t)N * N * sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(fields + (size_t)N * N, 0, (size_t)N * N * sizeof(double), s);
  if (e != cudaSuccess) return ECS_ERR_CUDA;
  // forcing spectrum on the box, mask[0,0] = False
  RowFwdParams<double> rf{}; rf.fields = fields; rf.H = H; rf.tw = tw; rf.B = 1;
  k_row_to_box<double, N, NA_XT><<<N / NA_XT, NA_XT * 32, na_smem_2f<N>(), s>>>(rf);
  ColBoxParams<double> cbp{}; cbp.H = H; cbp.V = fbox; cbp.tw = tw; cbp.vstride = 2L * K * M; cbp.B = 1; cbp.nf = 2;
  k_col_to_box<double, N><<<(2 * K + 3) / 4, 128, 0, s>>>(cbp);
  if (cudaMemsetAsync(fbox, 0, CB, s) != cudaSuccess) return ECS_ERR_CUDA;
  // state_vel: gather box, column inverse, row products, column forward, scatter
  const long nbox = (long)B * 2 * K * M;
  k_gather_box<double><<<(int)((nbox + 255) / 256), 256, 0, s>>>(f_hat, F, N, B);
  ColParams<double> cp{};
  cp.H = H; cp.G = G; cp.F = F; cp.A1 = nullptr; cp.K2 = nullptr; cp.OUT = OUT; cp.Etab = nullptr; cp.ctl = ctl;
  cp.fhat = fbox; cp.tw = tw; cp.nu = nu; cp.eta = eta; cp.B = B; cp.stage = COL_START; cp.produce = 1;
  cp.diss = 0; cp.rec = nullptr; cp.rec_bstride = 0;
  const int cols = B * K * 2;   // one warp per (batch, ky, channel)
  k_col_rk4<double, N, COL_START><<<(cols + 3) / 4, 128, 0, s>>>(cp);
  RowParams<double> rp{};
  rp.G = G; rp.H = H; rp.ctl = nullptr; rp.phys = nullptr; rp.phys_bstride = 0;
  rp.tw = tw; rp.b0x = b0x; rp.b0y = b0y; rp.B = B;
  k_row_rhs<double, N, NA_XT><<<B * (N / NA_XT), NA_XT * 32, na_smem_rhs<N>(), s>>>(rp);
  cp.stage = COL_PLAIN; cp.produce = 0; cp.diss = diss;
  k_col_rk4<double, N, COL_PLAIN><<<(cols + 3) / 4, 128, 0, s>>>(cp);
  const long nfull = (long)B * 2 * N * (N / 2 + 1);
  k_scatter_box<double><<<(int)((nfull + 255) / 256), 256, 0, s>>>(OUT, dfdt, N, B);
  return cudaGetLastError() == cudaSuccess ? ECS_OK : ECS_ERR_CUDA;
}

}  // namespace

extern "C" int ecs_state_vel_noalloc(int n, double nu, double eta, double b0x, double b0y, const double* forcing,
                                     const void* f_hat, void* dfdt_hat, int batch, int include_dissipation,
                                     void* stream) {
  if (!forcing || !f_hat || !dfdt_hat) return ECS_ERR_INVALID;
  if (batch < 1) return ECS_ERR_INVALID;
  if (n != 64 && n != 128) return ECS_ERR_TOO_LARGE;
  if (batch > NA_MAX_BATCH) return ECS_ERR_TOO_LARGE;
  unsigned char* base = nullptr;
  const int st = na_setup(&base);
  if (st) return st;
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 64)
    return na_state_vel<64>(base, nu, eta, b0x, b0y, forcing, (const double2*)f_hat, (double2*)dfdt_hat, batch,
                            include_dissipation, s);
  return na_state_vel<128>(base, nu, eta, b0x, b0y, forcing, (const double2*)f_hat, (double2*)dfdt_hat, batch,
                           include_dissipation, s);
}
