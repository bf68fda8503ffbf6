// Adaptive Lawson-RK4(3) ("EARK43") stepper, device resident.
//
// Reference: lawson_rk43 (jax_scripts/lib/timestepping.py:151-335).  One
// attempted step is five column launches (A..E) interleaved with four RHS row
// launches and one error row launch; the error reduction's last block performs
// the accept/reject decision and the step-size update on the device, so no host
// round trip happens per attempt.  Candidates that completed (|s-1| < 1e-10)
// skip all work, as the reference's lax.cond(complete, identity, do_step) does.
#pragma once

#include "kernels.cuh"

namespace ecs {

// Per-candidate state slots of the stepper, each a box vector [2][K][M].
// S_E holds (e, e L h/2) of the current attempt, e = exp(t L h/2) (written at
// stage A, read at stage C).
enum Rk43Slot { S_X0 = 0, S_K1, S_XE, S_K1E, S_K2, S_K3, S_X2, S_K4, S_XF, S_K5, S_E, S_NSLOT };
// Trajectory record per attempt (primal values needed by tangent/adjoint):
// start state, carried k1 (before twiddles), k2..k5, the stage inputs, and the
// attempt's integrating factor as (e, e L h/2) with e = exp(t L h/2), computed
// once here so that the tangent and adjoint passes do not recompute it per
// tangent (the same expression, so the same values).
enum Rk43Rec { RR_X0 = 0, RR_K1, RR_K2, RR_K3, RR_K4, RR_K5, RR_Y2, RR_Y3, RR_Y4, RR_XF, RR_E, RR_NREC };

enum Rk43Stage : int {
  R43_START = 6,  // no RHS input; inverse transforms of x0
  R43_INIT = 0,   // RHS of x0 finished: k1 = t v(x0)
  R43_A = 1,      // start of an attempt: promote accepted state, twiddle, input Y2
  R43_B = 2,      // k2 finished, input Y3
  R43_C = 3,      // k3 finished, twiddles, input Y4
  R43_D = 4,      // k4 finished, xf, input xf
  R43_E = 5,      // k5 finished, error field d = h (k5 - k4)/6 -> 2 inverse columns
};

template <typename R>
struct Col43Params {
  const cplx<R>* H;     // [B][NH][K][N]
  cplx<R>* G;           // [B][NG][K][N]
  cplx<R>* S;           // [B][S_NSLOT][2][K][M]
  StepCtl* ctl;         // [B]
  const cplx<R>* fhat;  // [K][M]
  const cplx<R>* tw;
  cplx<R>* rec;         // optional [B][cap][RR_NREC][2][K][M]
  int cap;
  R nu, eta;
  int B, stage;
};

// Slots (bits of Rk43Slot) that the algebra of an attempt stage reads after its
// forward transform; they are staged per column into shared memory.
__host__ __device__ constexpr unsigned r43_smask(int stage) {
  return stage == R43_B ? (1u << S_XE)
       : stage == R43_C ? (1u << S_XE) | (1u << S_K1E) | (1u << S_K2) | (1u << S_E)
       : stage == R43_D ? (1u << S_K1) | (1u << S_K2) | (1u << S_K3) | (1u << S_X2)
       : stage == R43_E ? (1u << S_K4) : 0u;
}
__host__ __device__ constexpr int popc_r43(unsigned m) { return m ? (int)(m & 1u) + popc_r43(m >> 1) : 0; }

// Slot rows staged per warp by an attempt stage (+ the forcing row), n <= 128.
template <int N, int STAGE> __host__ __device__ constexpr int col_rk43_nop() {
  return (N <= 128 && popc_r43(r43_smask(STAGE)) > 0) ? popc_r43(r43_smask(STAGE)) + 1 : 0;
}

// One warp's column `colid` of an attempt stage; `my_op` is the warp's staging
// buffer (col_rk43_nop rows of M entries).
template <typename R, int N, int STAGE>
__device__ __forceinline__ void col_rk43_body(const Col43Params<R>& p, int colid, int lane, const cplx<R>* s_tw,
                                              cplx<R>* my_op) {
  constexpr int E = N / 32;
  constexpr int KMAX = (N - 1) / 3, K = KMAX + 1, M = 2 * KMAX + 1;
  constexpr size_t VEC = (size_t)2 * K * M;
  const int ch = colid & 1, bk = colid >> 1, b = bk / K, ky = bk - b * K;   // one warp per (b, ky, channel)
  const StepCtl& c = p.ctl[b];
  if (c.done) return;
  const R t = (R)c.t, h = (R)c.h;
  const int pend = c.pending_accept;
  cplx<R>* S = p.S + (size_t)b * S_NSLOT * VEC;
  cplx<R>* rec = p.rec ? p.rec + ((size_t)b * p.cap + (c.attempts < p.cap ? c.attempts : p.cap - 1)) * RR_NREC * VEC
                       : nullptr;
  const bool has_rhs = STAGE != R43_A && STAGE != R43_START;
  // The slot rows (and, for the vorticity, the forcing row) that the algebra
  // reads after the forward transform, copied into the warp's shared buffer
  // with cp.async before it, so that their latency overlaps it (n <= 128).
  constexpr unsigned SM = N <= 128 ? r43_smask(STAGE) : 0u;
  constexpr int NS = popc_r43(SM), NOP = NS > 0 ? NS + 1 : 0;   // + the forcing row
  if constexpr (NOP > 0) {
    const size_t row = ((size_t)ch * K + ky) * M;
    int v = 0;
#pragma unroll
    for (int bit = 0; bit < 16; ++bit) {
      if ((SM >> bit) & 1u) {
        for (int s2 = lane; s2 < M; s2 += 32) cp_async_v(my_op + v * M + s2, S + bit * VEC + row + s2);
        ++v;
      }
    }
    if (ch == 0)
      for (int s2 = lane; s2 < M; s2 += 32) cp_async_v(my_op + NS * M + s2, p.fhat + ky * M + s2);
  }
  cplx<R> r[E];
  if (has_rhs) col_load_rhs<R, N>(p.H, b, ch, ky, lane, s_tw, r);
  if constexpr (NOP > 0) {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncwarp();
  }
  // staged (or, without staging, global) slot values at a slot
  auto SV = [&](int q, size_t o, int slot) -> cplx<R> {
    if constexpr (NOP > 0) return my_op[popc_r43(SM & ((1u << q) - 1u)) * M + slot];
    else return S[q * VEC + o];
  };
  const R coeff = ch == 0 ? p.nu : p.eta;
  cplx<R> x[E];
#pragma unroll
  for (int j = 0; j < E; ++j) {
    x[j] = mk<R>(0, 0);
    const int slot = pos_to_slot(spec_pos<N>(lane, j), N, KMAX, M);
    if (slot < 0) continue;
    const int kx = slot_to_kx(slot, KMAX, M);
    cplx<R> v = mk<R>(0, 0);
    if (has_rhs) {
      v = r[j];                                                        // zero at (0,0)
      if (ch == 0 && !(kx == 0 && ky == 0)) {
        if constexpr (NOP > 0) v = cadd(v, my_op[NS * M + slot]);
        else v = cadd(v, p.fhat[ky * M + slot]);
      }
    }
    const size_t o = ((size_t)ch * K + ky) * M + slot;
    const R L = diss_L<R>(kx, ky, coeff);
    const cplx<R> kv = cscale_rn(v, t);              // mod_vel_fn = t * vel_fn (timestepping.py:243)
    cplx<R> xin = mk<R>(0, 0);
    switch (STAGE) {
      case R43_START: xin = S[S_X0 * VEC + o]; break;
      case R43_INIT: S[S_K1 * VEC + o] = kv; break;
      case R43_A: {                                  // :266-270
        const cplx<R> xs = pend ? S[S_XF * VEC + o] : S[S_X0 * VEC + o];
        const cplx<R> ks = pend ? S[S_K5 * VEC + o] : S[S_K1 * VEC + o];
        if (pend) { S[S_X0 * VEC + o] = xs; S[S_K1 * VEC + o] = ks; }
        if (rec) { rec[RR_X0 * VEC + o] = xs; rec[RR_K1 * VEC + o] = ks; }
        const R e = exp((t * L) * h / R(2));         // e = exp(mod_L * h/2), not masked (:263)
        const cplx<R> eg = mk<R>(e, e * (L * h * R(0.5)));
        S[S_E * VEC + o] = eg;
        if (rec) rec[RR_E * VEC + o] = eg;
        const cplx<R> xe = cscale_rn(xs, e), k1e = cscale_rn(ks, e);
        S[S_XE * VEC + o] = xe; S[S_K1E * VEC + o] = k1e;
        xin = cadd(xe, cscale(cscale_rn(k1e, h), R(0.5)));
        if (rec) rec[RR_Y2 * VEC + o] = xin;
      } break;
      case R43_B: {                                  // :270-271
        S[S_K2 * VEC + o] = kv;
        if (rec) rec[RR_K2 * VEC + o] = kv;
        xin = cadd(SV(S_XE, o, slot), cscale(cscale_rn(kv, h), R(0.5)));
        if (rec) rec[RR_Y3 * VEC + o] = xin;
      } break;
      case R43_C: {                                  // :271-280
        if (rec) rec[RR_K3 * VEC + o] = kv;
        const R e = SV(S_E, o, slot).x;
        const cplx<R> x2 = cscale_rn(SV(S_XE, o, slot), e);
        const cplx<R> k1ee = cscale_rn(SV(S_K1E, o, slot), e);
        const cplx<R> k2e = cscale_rn(SV(S_K2, o, slot), e);
        const cplx<R> k3e = cscale_rn(kv, e);
        S[S_X2 * VEC + o] = x2; S[S_K1 * VEC + o] = k1ee;   // k1 carried on rejection is e^2 k1 (:297)
        S[S_K2 * VEC + o] = k2e; S[S_K3 * VEC + o] = k3e;
        xin = cadd_scaled_rn(x2, k3e, h);
        if (rec) rec[RR_Y4 * VEC + o] = xin;
      } break;
      case R43_D: {                                  // :280-281
        S[S_K4 * VEC + o] = kv;
        if (rec) rec[RR_K4 * VEC + o] = kv;
        const cplx<R> acc = cadd(cadd(cadd(cdiv_k<6>(SV(S_K1, o, slot)), cdiv_k<3>(SV(S_K2, o, slot))),
                                      cdiv_k<3>(SV(S_K3, o, slot))), cdiv_k<6>(kv));
        xin = cadd_scaled_rn(SV(S_X2, o, slot), acc, h);
        S[S_XF * VEC + o] = xin;
        if (rec) rec[RR_XF * VEC + o] = xin;
      } break;
      default: {                                     // R43_E: :282, :288
        S[S_K5 * VEC + o] = kv;
        if (rec) rec[RR_K5 * VEC + o] = kv;
        xin = cdiv_k<6>(cscale_rn(csub(kv, SV(S_K4, o, slot)), h));
      } break;
    }
    x[j] = xin;
  }
  if (STAGE == R43_INIT) return;
  if (STAGE == R43_E) col_inverse1<R, N>(x, p.G, NG, b, ch, ky, lane, s_tw, R(1) / (R(N) * R(N)));
  else col_inverse_uv<R, N>(x, p.G, b, ch, ky, lane, s_tw);
}

template <typename R, int N, int STAGE>
__global__ void __launch_bounds__(128) k_col_rk43(Col43Params<R> p) {
  constexpr int K = (N - 1) / 3 + 1, M = 2 * ((N - 1) / 3) + 1;
  constexpr int NOP = col_rk43_nop<N, STAGE>();
  __shared__ __align__(16) cplx<R> s_tw[fft_smem(N, 4)];
  __shared__ __align__(16) cplx<R> s_op[(NOP > 0 ? NOP : 1) * 4 * M];   // 4 warps per CTA
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int colid = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (colid >= p.B * K * 2) return;
  col_rk43_body<R, N, STAGE>(p, colid, lane, s_tw, s_op + (threadIdx.x >> 5) * NOP * M);
}

// Error norm max|irfft2(d)| of the two channels (timestepping.py:288-291) with
// the accept/reject decision and h update done by the last block of each
// candidate (timestepping.py:294-310).
template <typename R>
struct RowErrParams {
  const cplx<R>* G;     // [B][NG][K][N], fields 0,1 hold the inverse columns of d
  StepCtl* ctl;
  const cplx<R>* tw;
  double atol;
  double* rec_h;        // optional [B][cap] attempted step sizes ("hs", :239,:294)
  int* rec_acc;         // optional [B][cap] accept flags
  int cap;
  int B;
};

__device__ __forceinline__ void rk43_control(StepCtl& c, double atol, double err, double* rec_h, int* rec_acc) {
  const int a = c.attempts;
  const bool accept = err < atol;                          // :297 (false for NaN)
  if (rec_h) rec_h[a] = c.h;                               // :294
  if (rec_acc) rec_acc[a] = accept ? 1 : 0;
  if (accept) { c.s = c.s + c.h; c.accepted += 1; c.pending_accept = 1; }
  else { c.rejected += 1; c.pending_accept = 0; }
  c.fevals += 4;                                           // :285
  double hn = isnan(err) ? c.h / 2 : c.h * 0.9 * pow(atol / err, 0.25);   // :300-302
  const double ov = c.s + hn - 1.0;                        // :304-307 h - relu(s + h - 1)
  hn = hn - (isnan(ov) ? ov : (ov > 0.0 ? ov : 0.0));
  c.h = hn;
  c.err = err;
  c.attempts = a + 1;
  c.done = fabs(c.s - 1.0) < 1e-10 ? 1 : 0;                // :313
}

// max |irfft2(d)| over rows x0 .. x0 + XT - 1 of state b (the inverse column
// transforms of d in G fields 0 and 1), one warp per row; valid in thread 0.
template <typename R, int N, int XT>
__device__ __forceinline__ double row_err_max(const cplx<R>* G, int b, int x0, const cplx<R>* s_tw, cplx<R>* s_G,
                                              double* s_max) {
  constexpr int E = N / 32;
  constexpr int K = (N - 1) / 3 + 1;
  load_tile<R, N, XT>(s_G, G + (size_t)b * NG * K * N, 2 * K, x0);
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  cplx<R> z[E];
#pragma unroll
  for (int j = 0; j < E; ++j) z[j] = packed_pair<R, N, XT>(s_G, s_G + K * (XT + 1), lane + 32 * j, w);
  fft_dif<R, N, true>(z, s_tw, lane);
  double m = 0.0;
#pragma unroll
  for (int j = 0; j < E; ++j) {
    const double a = fabs((double)z[j].x), bb = fabs((double)z[j].y);
    m = (a > m || isnan(a)) ? a : m;
    m = (bb > m || isnan(bb)) ? bb : m;
  }
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const double q = __shfl_xor_sync(0xffffffffu, m, o);
    m = (q > m || isnan(q)) ? q : m;
  }
  if (lane == 0) s_max[w] = m;
  __syncthreads();
  double bm = s_max[0];
  for (int i = 1; i < XT; ++i) bm = (s_max[i] > bm || isnan(s_max[i])) ? s_max[i] : bm;
  return bm;
}

template <typename R, int N, int XT>
__global__ void __launch_bounds__(XT * 32) k_row_err(RowErrParams<R> p) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  cplx<R>* s_tw = reinterpret_cast<cplx<R>*>(smem_raw);
  cplx<R>* s_G = s_tw + fft_smem(N, XT);
  __shared__ double s_max[XT];
  __shared__ int s_last;
  const int tiles = N / XT;
  const int b = blockIdx.x / tiles, x0 = (blockIdx.x - b * tiles) * XT;
  pdl_trigger();
  load_twiddles<R, N>(s_tw, p.tw);
  pdl_wait();
  StepCtl& c = p.ctl[b];
  if (c.done) return;
  const double bm = row_err_max<R, N, XT>(p.G, b, x0, s_tw, s_G, s_max);
  if (threadIdx.x == 0) {
    // non-negative doubles (and NaN with the sign bit clear) order like their bit patterns
    atomicMax(&c.err_bits, (unsigned long long)__double_as_longlong(fabs(bm)));
    __threadfence();
    const unsigned prev = atomicAdd(&c.err_blocks, 1u);
    s_last = (prev == (unsigned)(tiles - 1));
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    const double err = __longlong_as_double((long long)atomicAdd(&c.err_bits, 0ull));
    const int a = c.attempts;
    rk43_control(c, p.atol, err, p.rec_h && a < p.cap ? p.rec_h + (size_t)b * p.cap : nullptr,
                 p.rec_acc && a < p.cap ? p.rec_acc + (size_t)b * p.cap : nullptr);
    c.err_bits = 0ull;
    c.err_blocks = 0u;
  }
}

// Initial control state: t = T, h = h0, s = 0 (timestepping.py:255).
static __global__ void k_rk43_setup(const double* T, double h0, StepCtl* ctl, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  StepCtl c;
  c.t = T[b]; c.h = h0; c.s = 0.0; c.err = 0.0;
  c.accepted = 0; c.rejected = 0; c.fevals = 1; c.done = 0;
  c.pending_accept = 0; c.attempts = 0; c.err_bits = 0ull; c.err_blocks = 0u; c.pad = 0;
  ctl[b] = c;
}

// Final state = x carried by the loop: xf if the last attempt was accepted.
template <typename R>
__global__ void k_rk43_resolve(cplx<R>* S, const StepCtl* ctl, cplx<R>* out, int n, int B) {
  const Geom g = make_geom(n);
  const size_t VEC = (size_t)2 * g.K * g.M;
  const long total = (long)B * VEC;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / VEC);
    const size_t o = i - (size_t)b * VEC;
    const cplx<R>* Sb = S + (size_t)b * S_NSLOT * VEC;
    out[i] = ctl[b].pending_accept ? Sb[S_XF * VEC + o] : Sb[S_X0 * VEC + o];
  }
}

static __global__ void k_count_done(const StepCtl* ctl, int* count, int B) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int s = 0;
    for (int b = 0; b < B; ++b) s += ctl[b].done;
    *count = s;
  }
}

}  // namespace ecs
