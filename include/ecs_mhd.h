/*
 * ecs_mhd.h -- C ABI of the B200-native hot path of mgolden30/ECS_MHD_2D.
 *
 * All array arguments are DEVICE pointers owned by the caller (e.g. torch
 * tensors' data_ptr()).  The library never frees caller memory.  Every call is
 * ordered on the caller's cudaStream_t (passed as void*; NULL = legacy default
 * stream) and returns an ecs_status; ecs_last_error() gives the message.
 * A context is not thread-safe: use one context per host thread.
 *
 * Layouts (C order, `real` = double for ECS_F64, float for ECS_F32):
 *   fields   real  [batch][2][n][n]          (omega, j) in real space, x then y
 *   f_hat    cplx  [batch][2][n][n/2+1]      jnp.fft.rfft2 layout (kx fftfreq, ky >= 0)
 *   box      cplx  [batch][2][K][M]          dealiased modes only, see ecs_box_dims
 *   T, sx    double[batch]
 * Flat vectors follow jax.flatten_util.ravel_pytree order of the reference's
 * {"T","fields","sx"} dicts: [T, fields(2*n*n), sx].
 *
 * Each entry point names the reference function it replaces (paths relative to
 * the reference project root).
 */
#ifndef ECS_MHD_H
#define ECS_MHD_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ecs_ctx ecs_ctx;

enum { ECS_F64 = 0, ECS_F32 = 1 };

enum {
  ECS_OK = 0,
  ECS_ERR_INVALID = 1,       /* bad argument */
  ECS_ERR_CUDA = 2,          /* CUDA runtime error */
  ECS_ERR_BAD_MODE = 3,      /* unknown integration mode (loss_functions.py:86-88) */
  ECS_ERR_NOT_COMPLETED = 4, /* adaptive integration hit its step cap (timestepping.py:313,327) */
  ECS_ERR_OOM = 5,           /* device allocation failed */
  ECS_ERR_UNSUPPORTED = 6,   /* grid size / dtype not built */
  ECS_ERR_TOO_LARGE = 7      /* beyond the fixed scratch of ecs_state_vel_noalloc */
};

/* Integration modes of mismatch_RPO (jax_scripts/lib/loss_functions.py:48-88):
 * Lawson_RK4 :57-65, Lawson_RK43 :72-77, RK4 (classic, dissipation in the
 * right-hand side) :49-56, Lawson_RK6 (num_checkpoints = 1, ministeps =
 * param_dict["steps"]) :66-71, TDRK4 (two-derivative RK4) :78-85. */
enum { ECS_MODE_LAWSON_RK4 = 1, ECS_MODE_LAWSON_RK43 = 2, ECS_MODE_RK4 = 3, ECS_MODE_LAWSON_RK6 = 4,
       ECS_MODE_TDRK4 = 5 };

typedef struct {
  double nu, eta;          /* param_dict["nu"], ["eta"] */
  double b0x, b0y;         /* param_dict["b0"] mean magnetic field */
  const double* forcing;   /* HOST real [n][n] forcing on the grid of construct_domain, or NULL */
  double kolmogorov_amp;   /* used when forcing == NULL: amp * cos(kolmogorov_k * y) */
  int kolmogorov_k;
} ecs_params;

typedef struct {
  int mode;                /* ECS_MODE_* */
  int num_checkpoints;     /* Lawson_RK4: param_dict["num_checkpoints"] */
  int ministeps;           /* Lawson_RK4: param_dict["ministeps"] */
  int shift_reflect_ny;    /* param_dict["shift_reflect_ny"] */
  int rot;                 /* param_dict["rot"] */
  double atol;             /* Lawson_RK43: adaptive_dict["atol"] */
  double h0;               /* Lawson_RK43: initial step (loss_functions.py:77 uses 1e-2) */
  int max_steps_per_checkpoint; /* Lawson_RK43: adaptive_dict["max_steps_per_checkpoint"] */
  int checkpoints;         /* Lawson_RK43: adaptive_dict["checkpoints"] */
  int ckpt_every;          /* Lawson_RK4 linearisation: keep only every k-th state and recompute
                              segments of k steps in ecs_jvp / ecs_vjp (0 = record every step);
                              k = ministeps mirrors jax.checkpoint at loss_functions.py:63 */
} ecs_shoot_cfg;

typedef struct {
  int completed;           /* |s - 1| < 1e-10 (timestepping.py:313) */
  double s;
  int accepted, rejected, fevals;
} ecs_info;

/* Library version string. */
const char* ecs_version(void);

/* Number of kernels this context has launched so far (instrumentation). */
long long ecs_launch_count(const ecs_ctx* ctx);

/* Times `iters` launches of a tangent-pass kernel (0: row pass k_row_tan,
 * 1: column pass k_col_tan) on the workspace left by the last ecs_jvp call of
 * `batch` tangents; returns ms per launch and the kernel's algorithmic bytes
 * per launch (instrumentation for roofline reporting; no reference counterpart). */
int ecs_bench_kernel(ecs_ctx* ctx, int which, int batch, int iters, float* ms, double* bytes, void* stream);

/* Newton-GMRES matvecs of `batch` different candidates in one call: for each
 * candidate b the objective (objective_RPO, jax_scripts/lib/loss_functions.py:132-148)
 * and its JVP for one tangent, as `batch` separate jax.jvp(obj, (x_b,), (v_b,))
 * calls would give them (jax_scripts/lib/utils.py:108, once per Arnoldi step
 * of jax_scripts/newton.py:165).  Mode Lawson_RK4 only; cfgs[b] (HOST array)
 * gives candidate b's num_checkpoints, ministeps, shift_reflect_ny and rot, so
 * candidates may differ in horizon, T, sx and symmetry (not in grid, dtype or
 * physics, which the context fixes).  Forward mode: the primal solves and their
 * tangents step together and no trajectory is kept (the context's linearisation
 * is untouched; a slot pool on the context restarts).  Device arrays: fields,
 * dfields, out_fields (may be NULL), out_dfields [batch][2][n][n]; T, sx, dT,
 * dsx, out_dT, out_dsx [batch] (double).  batch <= max_batch. */
int ecs_jvp_multi(ecs_ctx* ctx, const ecs_shoot_cfg* cfgs, const void* fields, const double* T, const double* sx,
                  void* out_fields, const void* dfields, const double* dT, const double* dsx, void* out_dfields,
                  double* out_dT, double* out_dsx, int batch, void* stream);

/* loss_RPO and its gradient for `batch` different candidates in one call, as
 * `batch` separate jax.value_and_grad(loss_RPO) calls give them
 * (jax_scripts/adjoint_descent.py:91; loss_functions.py:99-111).  Mode
 * Lawson_RK4 only; cfgs[b] (HOST array) gives candidate b's num_checkpoints,
 * ministeps, shift_reflect_ny and rot.  The forward solves step together and
 * keep a state every SEG steps (SEG, at most 32, divides every candidate's
 * step count); the adjoint sweep runs backwards over one recomputed segment
 * at a time, aligned at each candidate's end.  Device arrays: fields,
 * g_fields [batch][2][n][n]; T, sx, loss, g_T, g_sx [batch] (double).  The
 * context's linearisation is untouched; a slot pool on the context restarts. */
int ecs_loss_grad_multi(ecs_ctx* ctx, const ecs_shoot_cfg* cfgs, const void* fields, const double* T,
                        const double* sx, double* loss, void* g_fields, double* g_T, double* g_sx, int batch,
                        void* stream);

/* In-step timing of the batched tangent kernels (instrumentation for roofline
 * reporting; no reference counterpart).  enable = 1: the following
 * ecs_linearize_jvp calls (adaptive mode, pipelined path) record CUDA events
 * around tangent group 0's row-pass and column-pass launches of every accepted
 * attempt, on that group's stream, so each launch is timed in the launch shape
 * of the real sweep (the other groups run beside it).  enable = 0: stop, wait
 * for those events and return the mean duration (ms) and count per kind, and
 * group 0's batch.  Output pointers are HOST memory and may be NULL. */
int ecs_kernel_timing(ecs_ctx* ctx, int enable, double* row_ms, int* row_n, double* col_ms, int* col_n,
                      int* group_batch);

/* Context with grid tables and workspace for grids n in {64,128,256}
 * (replaces mhd_jax.construct_domain, jax_scripts/lib/mhd_jax.py:20-94, and
 * dictionaryIO.recompute_grid_information, jax_scripts/lib/dictionaryIO.py:64-78).
 * Uses the current CUDA device. */
int ecs_ctx_create(int n, int dtype, const ecs_params* params, int max_batch, ecs_ctx** out);
int ecs_ctx_destroy(ecs_ctx* ctx);
const char* ecs_last_error(const ecs_ctx* ctx);
/* K = ky columns kept, M = kx slots kept by the 2/3 mask (mhd_jax.py:65-70). */
int ecs_box_dims(const ecs_ctx* ctx, int* K, int* M);

/* rfft2 restricted to the dealiased box (jnp.fft.rfft2 at loss_functions.py:45). */
int ecs_to_box(ecs_ctx* ctx, const void* fields, void* box, int batch, void* stream);
/* irfft2 of a box spectrum (jnp.fft.irfft2, e.g. loss_functions.py:107). */
int ecs_from_box(ecs_ctx* ctx, const void* box, void* fields, int batch, void* stream);
/* irfft2(mask * rfft2(fields)) (newton.py:211-214, adjoint_descent.py:111-114). */
int ecs_dealias(ecs_ctx* ctx, const void* fields, void* out, int batch, void* stream);

/* state_vel (jax_scripts/lib/mhd_jax.py:105-175) on the full rfft2 layout. */
int ecs_state_vel(ecs_ctx* ctx, const void* f_hat, void* dfdt_hat, int batch,
                  int include_dissipation, void* stream);

/* lawson_rk4 with the mask (jax_scripts/lib/timestepping.py:46-81) on the full
 * rfft2 layout, in place; L_diag = dissipation(param_dict). */
int ecs_lawson_rk4(ecs_ctx* ctx, void* f_hat, double t, int steps, int batch, void* stream);

/* Fixed-step integration in place of rfft2 states f_hat [batch][2][n][n/2+1]
 * over time t in `steps` steps with the right-hand side, dissipation and mask
 * of mismatch_RPO's `mode` (ECS_MODE_RK4, _LAWSON_RK4, _LAWSON_RK6, _TDRK4;
 * jax_scripts/lib/timestepping.py:17-149).  Modes outside the 2/3 box are
 * zeroed by the Lawson modes (masked integrating factor) and kept by RK4 and
 * TDRK4 (masked right-hand side), as the reference does.  generate_turbulence.py
 * drives Lawson_RK6 this way (:88, :105). */
int ecs_integrate(ecs_ctx* ctx, int mode, void* f_hat, double t, int steps, int batch, void* stream);

/* Recurrence matrix of `snapshots` rfft2 states fs [snapshots][2][n][n/2+1]:
 * dist[j][i] = || |fs_j| - |fs_i| ||_2 (jax_scripts/generate_turbulence.py:136-146),
 * dist a DEVICE double [snapshots][snapshots]. */
int ecs_recurrence(ecs_ctx* ctx, const void* fs, int snapshots, double* dist, void* stream);

/* objective_RPO (jax_scripts/lib/loss_functions.py:132-148):
 * out_fields = irfft2(f0 - g.Phi_T(f0)), out_T = pt, out_sx = px (both 0 in value). */
int ecs_objective(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T,
                  const double* sx, void* out_fields, double* out_T, double* out_sx,
                  ecs_info* info, int batch, void* stream);

/* loss_RPO (jax_scripts/lib/loss_functions.py:99-111): mean(irfft2(f - f0)^2) per batch element. */
int ecs_loss(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T,
             const double* sx, double* loss, ecs_info* info, int batch, void* stream);

/* Linearise objective_RPO at one primal point (batch 1): runs the forward map
 * with a trajectory record kept in the context for later ecs_jvp/ecs_vjp calls
 * (replaces the primal half of jax.jvp / jax.vjp of objective_RPO,
 * jax_scripts/lib/utils.py:108, jax_scripts/newton.py:168).  out_fields
 * (optional) receives the objective's fields output. */
int ecs_linearize(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T,
                  const double* sx, void* out_fields, ecs_info* info, void* stream);

/* Jacobian-vector products of objective_RPO at the current linearisation for
 * `batch` tangents {dfields [batch][2][n][n], dT [batch], dsx [batch]}
 * (jac(primal, tangent), jax_scripts/lib/utils.py:108; the Newton-GMRES matvec). */
int ecs_jvp(ecs_ctx* ctx, const void* dfields, const double* dT, const double* dsx, void* out_dfields,
            double* out_dT, double* out_dsx, int batch, void* stream);

/* ecs_linearize and ecs_jvp in one call, as jax.jvp(obj, (x,), (v,)) returns
 * the objective and the Jacobian-vector products together
 * (jax_scripts/lib/utils.py:108).  In Lawson-RK4(3) mode the batch-1 primal
 * solve runs on a context-owned high-priority stream and the tangent sweep over
 * each completed chunk of attempts is queued on `stream` behind it, so the two
 * overlap; results equal ecs_linearize followed by ecs_jvp, and the
 * linearisation stays in the context for later ecs_jvp / ecs_vjp calls.
 * Requires stream to be the only stream using ctx during the call. */
int ecs_linearize_jvp(ecs_ctx* ctx, const ecs_shoot_cfg* cfg, const void* fields, const double* T,
                      const double* sx, void* out_fields, ecs_info* info, const void* dfields,
                      const double* dT, const double* dsx, void* out_dfields, double* out_dT,
                      double* out_dsx, int batch, void* stream);

/* Vector-Jacobian products of objective_RPO at the current linearisation for
 * `batch` cotangents {c_fields, c_T, c_sx}: gradients with respect to
 * {fields, T, sx} (jax.vjp(obj, input_dict), jax_scripts/newton.py:168-169;
 * with c_fields = out/n^2, c_T = c_sx = 0 it is the gradient of loss_RPO,
 * jax.value_and_grad at jax_scripts/adjoint_descent.py:91). */
int ecs_vjp(ecs_ctx* ctx, const void* c_fields, const double* c_T, const double* c_sx, void* g_fields,
            double* g_T, double* g_sx, int batch, void* stream);

/* One Arnoldi step's modified Gram-Schmidt in FP64 (jax_scripts/lib/linalg.py:65-86):
 * for j = 0..k: h_j = <w, Q[:,j]>, w -= h_j Q[:,j]; then Hcol[k+1] = |w| and
 * Q[:,k+1] = w / |w|.  Q is column-major with leading dimension ld >= len;
 * Hcol points at column k of H (k+2 entries written).  k = -1 only normalises
 * w into Q[:,0] (linalg.py:58) and writes |w| to Hcol[0].  len <= 131200. */
int ecs_arnoldi_mgs(double* Q, long ld, int k, const double* w, double* Hcol, long len, void* stream);

/* ecs_arnoldi_mgs followed by `reorth` (0..4) more sweeps j = 0..k that
 * subtract <w, Q[:,j]> Q[:,j] again without recording it, then the norm and
 * Q[:,k+1] = w/|w| (the twice-re-orthogonalised Arnoldi and Golub-Kahan steps
 * of newton_gmres_hookstep(_v2) and adjoint_GMRES, jax_scripts/lib/linalg.py:
 * 137-153, 254-266, 502-540). */
int ecs_arnoldi_mgs_reorth(double* Q, long ld, int k, const double* w, double* Hcol, long len, int reorth,
                           void* stream);

/* y = argmin |H y - b| for the (m+1) x m upper Hessenberg H (column-major,
 * leading dimension ldh >= m+1), m <= 128 (jnp.linalg.lstsq at linalg.py:93). */
int ecs_hessenberg_lstsq(const double* H, int ldh, int m, const double* b, double* y, void* stream);

/* Slot pool: continuous batching of Lawson_RK4 forward shootings
 * (objective_RPO / loss_RPO, loss_functions.py:99-148) over the context's
 * max_batch slots.  Each slot carries its own T, sx, symmetry and step count;
 * finished or empty slots are skipped by every launch, and new requests are
 * admitted between ecs_pool_advance calls while the others keep running.
 *   ecs_pool_reset   mark every slot empty
 *   ecs_pool_admit   load fields [2][n][n] (device) into an empty slot
 *   ecs_pool_advance advance all active slots by up to nsteps steps
 *   ecs_pool_poll    HOST arrays done[max_batch], steps_done[max_batch] (synchronises)
 *   ecs_pool_retire  residual irfft2(f0 - g.Phi_T(f0)) [2][n][n] and/or loss of a
 *                    finished slot (device pointers; either may be NULL); frees it */
int ecs_pool_reset(ecs_ctx* ctx, void* stream);
int ecs_pool_admit(ecs_ctx* ctx, int slot, const ecs_shoot_cfg* cfg, const void* fields, double T, double sx,
                   void* stream);
int ecs_pool_advance(ecs_ctx* ctx, int nsteps, void* stream);
int ecs_pool_poll(ecs_ctx* ctx, int* done, int* steps_done, void* stream);
int ecs_pool_retire(ecs_ctx* ctx, int slot, void* out_fields, double* loss, void* stream);

/* state_vel without any device allocation.  No counterpart in the reference.
 * For callers that cannot allocate device memory: a process whose GPU memory is
 * owned by another allocator (JAX/XLA preallocates most of the device and hands
 * buffers to custom calls, so a cudaMalloc from a library can fail there) or a
 * caller that forbids allocation after start-up.  Same computation and layout
 * as ecs_state_vel (FP64 complex f_hat / dfdt_hat [batch][2][n][n/2+1]); the
 * physics is passed directly, with `forcing` a DEVICE real [n][n] array on the
 * grid of construct_domain.  All scratch comes from one fixed ~3.8 MB device
 * array in the library, held on every GPU that loads it until exit.
 * Limits: n in {64, 128}, batch <= 4, else ECS_ERR_TOO_LARGE (batch < 1:
 * ECS_ERR_INVALID).  Calls share the array, so calls that overlap on the GPU
 * race; each call re-initialises what must start at zero.  The first call on a
 * device does a one-time synchronous set-up, so make it before any stream
 * capture; the device address it looks up is kept, which assumes the runtime's
 * primary context and no cudaDeviceReset afterwards. */
int ecs_state_vel_noalloc(int n, double nu, double eta, double b0x, double b0y, const double* forcing,
                          const void* f_hat, void* dfdt_hat, int batch, int include_dissipation, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ECS_MHD_H */
