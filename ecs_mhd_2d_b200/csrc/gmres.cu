// FP64 Arnoldi (modified Gram-Schmidt) and Hessenberg least squares for the
// matrix-free GMRES of the reference (jax_scripts/lib/linalg.py:12-98).
//
// ecs_arnoldi_mgs: one Arnoldi step's orthogonalisation (linalg.py:65-86):
//   for j = 0..k:  h_j = <w, q_j>;  w -= h_j q_j        (sequential, MGS)
//   h_{k+1} = |w|;  q_{k+1} = w / h_{k+1}
// runs on ONE thread-block cluster of 8 CTAs.  Each CTA keeps its slice of w in
// shared memory for the whole step; the per-j dot product is reduced across the
// cluster through distributed shared memory with hardware cluster barriers, in
// a fixed order (deterministic).  Q (column-major, leading dimension ld) is read
// once per column.
//
// ecs_hessenberg_lstsq: y = argmin |H y - b2| for the (m+1) x m upper
// Hessenberg H by Givens rotations in one CTA (linalg.py:92-93 uses lstsq; for
// full-rank H both give the same minimiser).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "../../include/ecs_mhd.h"

namespace cg = cooperative_groups;

namespace {

constexpr int CL = 8;          // CTAs per cluster
constexpr int TPB = 512;       // threads per CTA
constexpr int MAXSLICE = 16400; // doubles of w per CTA (128 KiB of shared memory)

__device__ double block_sum(double v, double* red) {
  for (int o = 16; o >= 1; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
    red[32] = s;
  }
  __syncthreads();
  s = red[32];
  __syncthreads();
  return s;
}

// reorth extra sweeps j = 0..k subtract the projections again without
// recording them (linalg.py:146-148, :260-262, :514-517, :534-537), before the norm.
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(TPB)
k_arnoldi_mgs(double* Q, long ld, int k, const double* w_in, double* Hcol, long len, int reorth) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  extern __shared__ double s_w[];
  __shared__ double red[33];
  __shared__ double part[2];          // this CTA's partial, read remotely by every CTA
  const long per = (len + CL - 1) / CL;
  const long lo = rank * per, hi = lo + per < len ? lo + per : len;
  const int cnt = (int)(hi > lo ? hi - lo : 0);
  for (int i = threadIdx.x; i < cnt; i += blockDim.x) s_w[i] = w_in[lo + i];
  __syncthreads();
  const int sweep = k + 1;                                  // projections per sweep
  const int total = sweep > 0 ? (reorth + 1) * sweep + 1 : 1;
  for (int it = 0; it < total; ++it) {
    const bool norm_pass = (it == total - 1);
    const int j = norm_pass ? k + 1 : it % sweep;
    const double* q = Q + (size_t)j * ld + lo;
    double v = 0.0;
    if (!norm_pass) for (int i = threadIdx.x; i < cnt; i += blockDim.x) v += s_w[i] * q[i];
    else for (int i = threadIdx.x; i < cnt; i += blockDim.x) v += s_w[i] * s_w[i];
    v = block_sum(v, red);
    if (threadIdx.x == 0) part[it & 1] = v;
    cluster.sync();
    // every CTA sums the partials in rank order (same value everywhere)
    double hj = 0.0;
    for (int r = 0; r < CL; ++r) hj += *cluster.map_shared_rank(&part[it & 1], r);
    if (!norm_pass) {
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) s_w[i] -= hj * q[i];
      if (it < sweep && rank == 0 && threadIdx.x == 0) Hcol[j] = hj;
    } else {
      const double nrm = sqrt(hj);
      if (rank == 0 && threadIdx.x == 0) Hcol[k + 1] = nrm;
      double* qn = Q + (size_t)(k + 1) * ld + lo;
      for (int i = threadIdx.x; i < cnt; i += blockDim.x) qn[i] = s_w[i] / nrm;
    }
    __syncthreads();
  }
  cluster.sync();   // no CTA exits while another may still read its shared partials
}

// Givens QR of the (m+1) x m upper Hessenberg H (column-major, ldh) and back
// substitution; H and b are copied to shared memory (m <= 128).
__global__ void k_hessenberg_lstsq(const double* H, int ldh, int m, const double* b, double* y) {
  extern __shared__ double sm[];
  double* h = sm;                       // (m+1) x m, column-major ld = m+1
  double* g = sm + (size_t)(m + 1) * m; // m+1
  const int ld = m + 1;
  for (int i = threadIdx.x; i < (m + 1) * m; i += blockDim.x) {
    const int r = i % ld, c = i / ld;
    h[i] = H[(size_t)c * ldh + r];
  }
  for (int i = threadIdx.x; i < m + 1; i += blockDim.x) g[i] = b[i];
  __syncthreads();
  __shared__ double cs, sn;
  for (int c = 0; c < m; ++c) {
    if (threadIdx.x == 0) {
      const double a = h[c * ld + c], bb = h[c * ld + c + 1];
      const double r = hypot(a, bb);
      cs = r == 0.0 ? 1.0 : a / r;
      sn = r == 0.0 ? 0.0 : bb / r;
    }
    __syncthreads();
    for (int cc = c + threadIdx.x; cc < m; cc += blockDim.x) {
      const double a = h[cc * ld + c], bb = h[cc * ld + c + 1];
      h[cc * ld + c] = cs * a + sn * bb;
      h[cc * ld + c + 1] = -sn * a + cs * bb;
    }
    if (threadIdx.x == 0) {
      const double a = g[c], bb = g[c + 1];
      g[c] = cs * a + sn * bb;
      g[c + 1] = -sn * a + cs * bb;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int r = m - 1; r >= 0; --r) {
      double s = g[r];
      for (int c = r + 1; c < m; ++c) s -= h[c * ld + r] * y[c];
      y[r] = s / h[r * ld + r];
    }
  }
}

}  // namespace

extern "C" int ecs_arnoldi_mgs(double* Q, long ld, int k, const double* w, double* Hcol, long len, void* stream) {
  return ecs_arnoldi_mgs_reorth(Q, ld, k, w, Hcol, len, 0, stream);
}

extern "C" int ecs_arnoldi_mgs_reorth(double* Q, long ld, int k, const double* w, double* Hcol, long len, int reorth,
                                      void* stream) {
  if (!Q || !w || !Hcol || k < -1 || len < 1 || ld < len || reorth < 0 || reorth > 4) return ECS_ERR_INVALID;
  const long per = (len + CL - 1) / CL;
  if (per > MAXSLICE) return ECS_ERR_UNSUPPORTED;
  const size_t smem = (size_t)per * sizeof(double);
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(k_arnoldi_mgs, cudaFuncAttributeMaxDynamicSharedMemorySize, MAXSLICE * 8) != cudaSuccess)
      return ECS_ERR_CUDA;
    configured = true;
  }
  k_arnoldi_mgs<<<CL, TPB, smem, (cudaStream_t)stream>>>(Q, ld, k, w, Hcol, len, reorth);
  return cudaGetLastError() == cudaSuccess ? ECS_OK : ECS_ERR_CUDA;
}

extern "C" int ecs_hessenberg_lstsq(const double* H, int ldh, int m, const double* b, double* y, void* stream) {
  if (!H || !b || !y || m < 1 || m > 128 || ldh < m + 1) return ECS_ERR_INVALID;
  const size_t smem = ((size_t)(m + 1) * m + m + 1) * sizeof(double);
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(k_hessenberg_lstsq, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024) != cudaSuccess)
      return ECS_ERR_CUDA;
    configured = true;
  }
  k_hessenberg_lstsq<<<1, 256, smem, (cudaStream_t)stream>>>(H, ldh, m, b, y);
  return cudaGetLastError() == cudaSuccess ? ECS_OK : ECS_ERR_CUDA;
}
