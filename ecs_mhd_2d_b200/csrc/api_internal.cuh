// Host-side context shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "../../include/ecs_mhd.h"

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
  long long launches = 0;           // kernels launched through this context
  int pdl = 1;                      // stepping kernels use programmatic dependent launch (ECS_PDL=0 disables)
  int rowtan_xt = 4;                // rows per CTA of the batched tangent row pass at n = 128 (ECS_ROWTAN_XT=4 or 8; 4 measured best)
  int pdl_minb = 1;                 // smallest batch launched with programmatic dependent launch (ECS_PDL_MINB)
  int plain_order = 0;              // depth of PlainOrder scopes (no programmatic launch below batch 8)
  int tgroups = 3;                  // tangent groups of ecs_linearize_jvp (ECS_TGROUPS=1..4; 3 measured best at B=64)
  int regen_items = 0;              // stage inputs per regeneration chunk (ECS_REGEN_ITEMS, at least 8; 0: about 384 MiB)
  // Cluster-resident chains (k_tan_chain for the adaptive tangent sweep,
  // k_rk4_chain for Lawson-RK4 stepping) run batches up to the number of
  // 16-warp clusters the device holds at once; batches up to the number of
  // 8-warp clusters (16 CTAs each at n = 128) use those.  Measured at n = 128
  // FP64 (matvecs/s, state-steps/s; launch per pass -> chain): batch 1 11.2 ->
  // 12.5 and 23.4k -> 30.1k, batch 4 30.3 -> 50.5 and 67.5k -> 120k, batch 8
  // 59.4 -> 68.7 and 111k -> 165k; at batch 16 the launch-per-pass path is ahead.
  int chain_res8 = 0, chain_res16 = 0;   // clusters of each shape the device holds at once (set at creation)
  int chain_w = 0;                  // warps per CTA forced for the chains (ECS_CHAIN_WARPS=8 or 16; 0: by batch as above)
  int chain_dsh = 1;                // the 8-warp tangent chain keeps each column's tangent slots in shared memory (ECS_CHAIN_DSLOTS=0: global)
  int chain_dsm = -1;               // G / H exchange of the chains: 1 distributed shared memory, 0 global memory (ECS_CHAIN_DSMEM; -1: global for the tangent chain, shared for Lawson-RK4, as measured)
  int chain_minb = 1, chain_maxb = -1;         // batch range of the tangent chain (ECS_CHAIN_MINB / ECS_CHAIN_MAXB; -1: chain_res16; 0: off)
  int rk4chain_minb = 1, rk4chain_maxb = -1;   // batch range of the Lawson-RK4 chain (ECS_RK4CHAIN_MINB / ECS_RK4CHAIN_MAXB)
  int rk43chain_minb = 1, rk43chain_maxb = -1; // batch range of the adaptive Lawson-RK4(3) solve's chain (ECS_RK43CHAIN_MINB / _MAXB)
  // linearisation (primal trajectory record) shared by JVP / VJP calls
  struct Lin {
    int valid = 0, mode = 0;
    ecs_shoot_cfg cfg{};
    double T = 0, sx = 0, h = 0;
    long nrec = 0;                  // Lawson-RK4: steps; Lawson-RK4(3): attempts
    std::vector<int> acc;           // Lawson-RK4(3) accept flags
    std::vector<double> hs;         // Lawson-RK4(3) attempted step sizes
    void* rec = nullptr; size_t rec_bytes = 0;
    void* phi = nullptr;            // final primal box state
    void* f0box = nullptr;          // box(rfft2(fields))
    void* vt = nullptr;             // irfft2(state_vel(f0, dissipation)) [2][N][N]
    void* vx = nullptr;             // irfft2(i kx f0)                    [2][N][N]
    double* dsx = nullptr;          // primal sx on the device
    double* dT = nullptr;           // primal T on the device
    double* rec_h = nullptr; int* rec_acc = nullptr; size_t cap = 0;
    long seg = 0;                   // Lawson-RK4 checkpoint interval (0: full record)
    void* ckpt = nullptr; size_t ckpt_bytes = 0;   // segment start states
    void* rec2 = nullptr; size_t rec2_bytes = 0;   // second segment record (pipelined adjoint)
  } lin;
  // tangent / adjoint workspace (grown on demand)
  void* D = nullptr; size_t D_bytes = 0;          // tangent or adjoint slots
  void* Greg = nullptr; void* Phys = nullptr; size_t reg_items = 0;   // regenerated primal fields
  long* items = nullptr; size_t items_cap = 0;
  void* chain_ops = nullptr; size_t chain_ops_bytes = 0;   // pass list of the cluster-resident tangent sweep
  double* hacc = nullptr; size_t hacc_bytes = 0;   // adjoint dL/dh accumulators [B][K]
  // CUDA graph of a chunk of adaptive attempts (replayed on the caller's stream)
  cudaStream_t cap_stream = nullptr;
  struct Graph43 {
    cudaGraphExec_t exec = nullptr;
    int B = 0, cap = 0;
    double atol = 0;
    void* rec = nullptr; double* rec_h = nullptr; int* rec_acc = nullptr;
    void* G = nullptr; void* H = nullptr;   // scratch the captured kernels use
    long long nodes = 0;
  } g43;
  // pipelined linearisation + JVP (ecs_linearize_jvp): the batch-1 primal runs on
  // a high-priority stream with its own scratch while the tangents run on the
  // caller's stream; per chunk of attempts the primal's control block and
  // accept flags come back through double-buffered pinned memory
  cudaStream_t pstream = nullptr;
  cudaEvent_t pev[2] = {nullptr, nullptr};
  void* Gp = nullptr; void* Hp = nullptr;   // [NG][K][N], [NHA][K][N] primal scratch (batch 1)
  void* Gx = nullptr; size_t Gx_bytes = 0;  // TDRK4 tangent/adjoint: second G array [B][NG][K][N]
  static constexpr int MAXG = 4;            // tangent groups of ecs_linearize_jvp
  cudaStream_t tstream[MAXG] = {};          // streams of groups 1.. (group 0 uses the caller's stream)
  cudaEvent_t tfork = nullptr, tjoin[MAXG][2] = {};
  ecs::StepCtl* hctl = nullptr;             // pinned [2]
  int* hchunk_acc = nullptr;                // pinned [2][16]
  double* hchunk_h = nullptr;               // pinned [2][16]
  long* hitems = nullptr; size_t hitems_cap = 0;   // pinned staging of regeneration items
  // slot pool (continuous batching of forward shootings)
  struct PoolSlot { int active = 0, ny = 0, rot = 0; long steps = 0; };
  std::vector<PoolSlot> pool;
  void* pool_fields = nullptr;   // [B][2][N][N] the admitted fields (residual base)
  double* pool_sx = nullptr;     // [B]
  struct GraphPool { cudaGraphExec_t exec = nullptr; long long nodes = 0; } gpool;
  struct Graph4 {
    cudaGraphExec_t exec = nullptr;
    int B = 0;
    long long nodes = 0;
  } g4;
  // 16-step graphs of the other fixed-step modes (RK4, Lawson-RK6, TDRK4)
  struct GraphFx { cudaGraphExec_t exec = nullptr; int B = 0; void* phys = nullptr; long long nodes = 0; } gfx[3];
  void* fxphys = nullptr; size_t fxphys_bytes = 0;   // TDRK4: recorded u, v, B_x, B_y per batch element
  // several candidates' Lawson-RK4 matvecs in one forward-mode sweep
  // (ecs_jvp_multi): the tangents' own G/H, the primal physical fields of the
  // current stage, the current step's record, the phase fields, dT scales
  struct Multi {
    void* G = nullptr; void* H = nullptr; void* phys = nullptr; void* rec = nullptr;
    void* vt = nullptr; void* vx = nullptr; double* dscale = nullptr; double* dT = nullptr;
    // the 8-step graph bakes in B and the tangent-slot buffer D (which grows)
    struct Graph { cudaGraphExec_t exec = nullptr; int B = 0; void* D = nullptr; long long nodes = 0; } g;
    // several candidates' gradients (ecs_loss_grad_multi): segment start states,
    // one segment's record and stage fields, residuals, per-candidate segment counts
    void* ckpt = nullptr; size_t ckpt_bytes = 0;
    void* grec = nullptr; size_t grec_bytes = 0;
    void* gphys = nullptr; size_t gphys_bytes = 0;
    void* res = nullptr; size_t res_bytes = 0;
    int* nseg = nullptr;
  } mj;
  // in-step timing of the batched tangent kernels (ecs_kernel_timing): CUDA
  // events around tangent group 0's row-pass and column-pass launches inside
  // the attempt loop of ecs_linearize_jvp, on that group's stream
  struct KernelTiming {
    int on = 0, batch = 0;
    std::vector<cudaEvent_t> ev;    // event pool, created on demand
    std::vector<int> kind;          // per recorded pair: 0 row pass, 1 column pass
    size_t used = 0;                // events recorded (two per pair)
  } kt;
  std::string err;
};

namespace ecs {

template <int N> struct Geomc {
  static constexpr int kmax = (N - 1) / 3;
  static constexpr int K = kmax + 1;
  static constexpr int M = 2 * kmax + 1;
};

int set_err(ecs_ctx* c, int code, const std::string& msg);
// Held by every CUDA graph capture (begin to instantiate) and by context
// creation and destruction, whose set-up synchronises the device: a
// device-wide synchronisation while another thread captures is an error.
std::mutex& capture_mutex();
int cuda_err(ecs_ctx* c, cudaError_t e, const char* where);
// Kernel timing marks (no-ops unless ecs_kernel_timing enabled them): an event
// before a launch, and one after it naming its kind (0 row pass, 1 column pass).
void kt_begin(ecs_ctx* c, cudaStream_t s);
void kt_end(ecs_ctx* c, int kind, int batch, cudaStream_t s);
void* dev_alloc(ecs_ctx* c, size_t bytes, int* st);
// (re)allocate a growable device buffer owned by the context (not in allocs)
int grow(ecs_ctx* c, void** p, size_t* have, size_t need);

static __global__ void k_fill(double* p, double v, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}

}  // namespace ecs
